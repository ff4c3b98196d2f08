// Drop-in definitions of gtom's RELION-path functions over this library's C
// ABI (include/gtomrln.h).
//
// A maintainer of a gtom-based code (Warp's native layer, gtom's own
// SubTomograms.cu, the MEX front-end) compiles this file instead of the
// reference's src/Relion/{Project,Backproject,ProjectShifted,
// BackprojectShifted,BackprojectTomo,ConvertWeights,DiffRemap,Misc,
// StoreWeights}.cu and the d_ReconstructGridding definition of
// src/Reconstruction/RecFourier.cu, against gtom's own headers, and links
// libgtomrln.so.  Every definition has the signature declared in gtom's
// include/Relion.cuh and include/Reconstruction.cuh, so the mangled symbols
// are the reference's and no call site changes (checked by
// tests/test_shim_cpu.py against the reference's own objects).
//
//   nvcc -std=c++14 -c gtom_rln_shim.cu -I<gtom>/include -I<this repo>/include
//
// Semantics kept: work is ordered on the legacy default stream (stream 0),
// like the reference's launches; results land in the caller's buffers with
// the reference's layouts.  Where the reference calls `throw;` (which ends
// the process) or its cuFFT wrapper throws, these throw std::runtime_error
// with the library's message instead.
#include <stdexcept>
#include <string>

#include "Prerequisites.cuh"
#include "Angles.cuh"  // glm::mat3, as the reference's own Relion sources include it
#include "Reconstruction.cuh"
#include "Relion.cuh"
#include "gtomrln.h"

namespace {
void check(int status, const char* what) {
  if (status != GTOMRLN_OK) throw std::runtime_error(std::string(what) + ": " + gtomrln_last_error());
}
const float* cf(const void* p) { return static_cast<const float*>(p); }
float* f(void* p) { return static_cast<float*>(p); }
}  // namespace

namespace gtom {

// ------------------------------------------------------------ Project.cu --
// include/Relion.cuh:34, src/Relion/Project.cu:12-23
void d_rlnProject(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj, tfloat3* h_angles,
                  float supersample, uint batch) {
  check(gtomrln_project_angles(cf(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj), dimsproj.x,
                               dimsproj.y, dimsproj.z, cf(h_angles), supersample, batch, nullptr),
        "d_rlnProject");
}

// include/Relion.cuh:35, src/Relion/Project.cu:25-43
void d_rlnProject(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj, uint rmax,
                  glm::mat3* d_matrices, uint batch) {
  check(gtomrln_project(cf(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj), dimsproj.x,
                        dimsproj.y, dimsproj.z, rmax, cf(d_matrices), batch, nullptr),
        "d_rlnProject");
}

// include/Relion.cuh:36, src/Relion/Project.cu:45-56
void d_rlnProject(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj,
                  tfloat3* h_angles, float supersample, uint batch) {
  check(gtomrln_project_tex_angles(t_volumeRe, t_volumeIm, dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj),
                                   dimsproj.x, dimsproj.y, dimsproj.z, cf(h_angles), supersample, batch,
                                   nullptr),
        "d_rlnProject");
}

// include/Relion.cuh:37, src/Relion/Project.cu:58-87
void d_rlnProject(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj,
                  uint rmax, glm::mat3* d_matrices, uint batch) {
  check(gtomrln_project_tex(t_volumeRe, t_volumeIm, dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj),
                            dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(d_matrices), batch, nullptr),
        "d_rlnProject");
}

// --------------------------------------------------------- Backproject.cu --
// include/Relion.cuh:9, src/Relion/Backproject.cu:48-124
void d_rlnBackproject(tcomplex* d_volumeft, tfloat* d_volumeweights, int3 dimsvolume, tcomplex* d_projft,
                      tfloat* d_projweights, int3 dimsproj, uint rmax, glm::mat3* d_matrices, int* d_ivolume,
                      float4 magnification, float ewaldradiussuper, bool outputdecentered,
                      bool squareinterpweights, uint batch) {
  check(gtomrln_backproject(f(d_volumeft), d_volumeweights, dimsvolume.x, dimsvolume.y, dimsvolume.z,
                            cf(d_projft), d_projweights, dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(d_matrices),
                            d_ivolume, magnification.x, magnification.y, magnification.z, magnification.w,
                            ewaldradiussuper, outputdecentered, squareinterpweights, batch, nullptr),
        "d_rlnBackproject");
}

// include/Relion.cuh:10, src/Relion/Backproject.cu:23-46
void d_rlnBackproject(tcomplex* d_volumeft, tfloat* d_volumeweights, int3 dimsvolume, tcomplex* d_projft,
                      tfloat* d_projweights, int3 dimsproj, uint rmax, tfloat3* h_angles, int* h_ivolume,
                      float4 magnification, float ewaldradius, float supersample, bool outputdecentered,
                      bool squareinterpweights, uint batch) {
  check(gtomrln_backproject_angles(f(d_volumeft), d_volumeweights, dimsvolume.x, dimsvolume.y, dimsvolume.z,
                                   cf(d_projft), d_projweights, dimsproj.x, dimsproj.y, dimsproj.z, rmax,
                                   cf(h_angles), h_ivolume, magnification.x, magnification.y, magnification.z,
                                   magnification.w, ewaldradius, supersample, outputdecentered,
                                   squareinterpweights, batch, nullptr),
        "d_rlnBackproject");
}

// ----------------------------------------------------- BackprojectTomo.cu --
// include/Relion.cuh:13, src/Relion/BackprojectTomo.cu:11-28
void d_BackprojectTomo(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_projft, tfloat* d_projweights,
                       int3 dimsproj, uint rmax, tfloat3* h_angles, uint batch) {
  check(gtomrln_backproject_tomo_angles(f(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, cf(d_projft),
                                        d_projweights, dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(h_angles),
                                        batch, nullptr),
        "d_BackprojectTomo");
}

// include/Relion.cuh:14, src/Relion/BackprojectTomo.cu:30-46
void d_BackprojectTomo(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_projft, tfloat* d_projweights,
                       int3 dimsproj, uint rmax, glm::mat3* d_matrices, uint batch) {
  check(gtomrln_backproject_tomo(f(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, cf(d_projft),
                                 d_projweights, dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(d_matrices), batch,
                                 nullptr),
        "d_BackprojectTomo");
}

// -------------------------------------------------- BackprojectShifted.cu --
// include/Relion.cuh:17, src/Relion/BackprojectShifted.cu:11-35
void d_rlnBackprojectShifted(tcomplex* d_volumeft, tfloat* d_volumeweights, int3 dimsvolume, tcomplex* d_projft,
                             tfloat* d_projweights, int3 dimsproj, uint rmax, tfloat3* h_angles, tfloat3* h_shifts,
                             float* h_globalweights, float supersample, uint batch) {
  check(gtomrln_backproject_shifted_angles(f(d_volumeft), d_volumeweights, dimsvolume.x, dimsvolume.y,
                                           dimsvolume.z, cf(d_projft), d_projweights, dimsproj.x, dimsproj.y,
                                           dimsproj.z, rmax, cf(h_angles), cf(h_shifts), h_globalweights,
                                           supersample, batch, nullptr),
        "d_rlnBackprojectShifted");
}

// include/Relion.cuh:18, src/Relion/BackprojectShifted.cu:37-58
void d_rlnBackprojectShifted(tcomplex* d_volumeft, tfloat* d_volumeweights, int3 dimsvolume, tcomplex* d_projft,
                             tfloat* d_projweights, int3 dimsproj, uint rmax, glm::mat3* d_matrices,
                             tfloat3* d_shifts, float* d_globalweights, uint batch) {
  check(gtomrln_backproject_shifted(f(d_volumeft), d_volumeweights, dimsvolume.x, dimsvolume.y, dimsvolume.z,
                                    cf(d_projft), d_projweights, dimsproj.x, dimsproj.y, dimsproj.z, rmax,
                                    cf(d_matrices), cf(d_shifts), d_globalweights, batch, nullptr),
        "d_rlnBackprojectShifted");
}

// ------------------------------------------------------ ProjectShifted.cu --
// include/Relion.cuh:40, src/Relion/ProjectShifted.cu:32-56
void d_rlnProjectShifted(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj,
                         tfloat3* h_angles, tfloat3* h_shifts, float* h_globalweights, float supersample,
                         uint batch) {
  check(gtomrln_project_shifted_angles(cf(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj),
                                       dimsproj.x, dimsproj.y, dimsproj.z, cf(h_angles), cf(h_shifts),
                                       h_globalweights, supersample, batch, nullptr),
        "d_rlnProjectShifted");
}

// include/Relion.cuh:41, src/Relion/ProjectShifted.cu:58-75
void d_rlnProjectShifted(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj, int3 dimsproj, uint rmax,
                         glm::mat3* d_matrices, tfloat3* d_shifts, float* d_globalweights, uint batch) {
  check(gtomrln_project_shifted(cf(d_volumeft), dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj),
                                dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(d_matrices), cf(d_shifts),
                                d_globalweights, batch, nullptr),
        "d_rlnProjectShifted");
}

// include/Relion.cuh:42, src/Relion/ProjectShifted.cu:78-101
void d_rlnProjectShifted(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume, tcomplex* d_proj,
                         int3 dimsproj, tfloat3* h_angles, tfloat3* h_shifts, float* h_globalweights,
                         float supersample, uint batch) {
  check(gtomrln_project_shifted_tex_angles(t_volumeRe, t_volumeIm, dimsvolume.x, dimsvolume.y, dimsvolume.z,
                                           f(d_proj), dimsproj.x, dimsproj.y, dimsproj.z, cf(h_angles),
                                           cf(h_shifts), h_globalweights, supersample, batch, nullptr),
        "d_rlnProjectShifted");
}

// include/Relion.cuh:43, src/Relion/ProjectShifted.cu:103-122
void d_rlnProjectShifted(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume, tcomplex* d_proj,
                         int3 dimsproj, uint rmax, glm::mat3* d_matrices, tfloat3* d_shifts,
                         float* d_globalweights, uint batch) {
  check(gtomrln_project_shifted_tex(t_volumeRe, t_volumeIm, dimsvolume.x, dimsvolume.y, dimsvolume.z, f(d_proj),
                                    dimsproj.x, dimsproj.y, dimsproj.z, rmax, cf(d_matrices), cf(d_shifts),
                                    d_globalweights, batch, nullptr),
        "d_rlnProjectShifted");
}

// ------------------------------------------------------ ConvertWeights.cu --
// include/Relion.cuh:21
void d_rlnConvertWeightsDense(tfloat* d_weights, uint nparticles, uint nclasses, uint nrot, uint ntrans,
                              tfloat* d_pdfrot, tfloat* d_pdftrans, tfloat* d_mindiff2) {
  check(gtomrln_convert_weights_dense(d_weights, nparticles, nclasses, nrot, ntrans, d_pdfrot, d_pdftrans,
                                      d_mindiff2, nullptr),
        "d_rlnConvertWeightsDense");
}

// include/Relion.cuh:22
void d_rlnConvertWeightsSparse(tfloat* d_weightsdense, tfloat* d_weightssparse, uint4* d_combinations,
                               uint nsparse, uint nrot, uint ntrans, tfloat* d_pdfrot, tfloat* d_pdftrans,
                               tfloat* d_mindiff2) {
  check(gtomrln_convert_weights_sparse(d_weightsdense, d_weightssparse, reinterpret_cast<const unsigned*>(d_combinations),
                                       nsparse, nrot, ntrans, d_pdfrot, d_pdftrans, d_mindiff2, nullptr),
        "d_rlnConvertWeightsSparse");
}

// include/Relion.cuh:23
void d_rlnConvertWeightsSort(tfloat* d_input, uint n) {
  check(gtomrln_convert_weights_sort(d_input, n, nullptr), "d_rlnConvertWeightsSort");
}

// include/Relion.cuh:24
void d_rlnConvertWeightsCompact(tfloat* d_input, tfloat* d_output, uint& n) {
  unsigned count = n;
  check(gtomrln_convert_weights_compact(d_input, d_output, &count, nullptr), "d_rlnConvertWeightsCompact");
  n = count;
}

// ----------------------------------------------------------- DiffRemap.cu --
// include/Relion.cuh:27
void d_rlnDiffRemapDense(tfloat* d_input, tfloat* d_output, uint3* d_orientationindices, uint norientations,
                         uint iclass, uint nparticles, uint nclasses, uint nrot, uint ntrans, uint ntranspadded,
                         tfloat* d_xi2imgs, tfloat* d_sqrtxi2, bool docc) {
  check(gtomrln_diff_remap_dense(d_input, d_output, reinterpret_cast<const unsigned*>(d_orientationindices),
                                 norientations, iclass, nparticles, nclasses, nrot, ntrans, ntranspadded, d_xi2imgs,
                                 d_sqrtxi2, docc, nullptr),
        "d_rlnDiffRemapDense");
}

// include/Relion.cuh:28
void d_rlnDiffRemapSparse(tfloat* d_input, tfloat* d_output, tfloat* d_mindiff2, uint3* d_combinations,
                          uint* d_hiddenover, uint elements, uint tileelements, uint weightsperpart, uint nparticles,
                          tfloat* d_xi2imgs, tfloat* d_sqrtxi2, bool docc) {
  check(gtomrln_diff_remap_sparse(d_input, d_output, d_mindiff2, reinterpret_cast<const unsigned*>(d_combinations),
                                  d_hiddenover, elements, tileelements, weightsperpart, nparticles, d_xi2imgs,
                                  d_sqrtxi2, docc, nullptr),
        "d_rlnDiffRemapSparse");
}

// ---------------------------------------------------------------- Misc.cu --
// include/Relion.cuh:31
void d_rlnCreateMinvsigma2s(tfloat* d_output, int* d_mresol, uint elements, tfloat* d_sigma2noise,
                            tfloat sigma2fudge) {
  check(gtomrln_create_minvsigma2s(d_output, d_mresol, elements, d_sigma2noise, sigma2fudge, nullptr),
        "d_rlnCreateMinvsigma2s");
}

// -------------------------------------------------- SquaredDifferences.cu --
// include/Relion.cuh:46 (declared by the reference, no definition in it)
void d_rlnSquaredDifferences(tcomplex* d_particleft, tfloat* d_minvsigma2, tfloat* d_ctf, int3 dimsparticle,
                             uint nparticles, tcomplex* d_precalcshifts, uint nshifts, tcomplex* d_refft, uint nrefs,
                             uint tile, tfloat* d_diff2, bool dofirstitercc) {
  check(gtomrln_squared_differences(cf(d_particleft), d_minvsigma2, d_ctf, dimsparticle.x, dimsparticle.y,
                                    dimsparticle.z, nparticles, cf(d_precalcshifts), nshifts, cf(d_refft), nrefs,
                                    tile, d_diff2, dofirstitercc, nullptr),
        "d_rlnSquaredDifferences");
}

// include/Relion.cuh:48 (declared by the reference, no definition in it)
void d_rlnSquaredDifferencesSparse(tcomplex* d_particleft, tfloat* d_minvsigma2, tfloat* d_ctf,
                                   int3 dimsparticle, tcomplex* d_precalcshifts, tcomplex* d_refft, tfloat* d_diff2,
                                   uint3* d_combination, uint ncombinations, uint groupsize, bool dofirstitercc) {
  check(gtomrln_squared_differences_sparse(cf(d_particleft), d_minvsigma2, d_ctf, dimsparticle.x, dimsparticle.y,
                                           dimsparticle.z, cf(d_precalcshifts), cf(d_refft), d_diff2,
                                           reinterpret_cast<const unsigned*>(d_combination), ncombinations,
                                           groupsize, dofirstitercc, nullptr),
        "d_rlnSquaredDifferencesSparse");
}

// -------------------------------------------------------- StoreWeights.cu --
// include/Relion.cuh:51-57
void d_rlnStoreWeightsAdd(tcomplex* d_input, tfloat* d_ctf, tcomplex* d_ref, tfloat* d_minvsigma2, int* d_mresol,
                          uint elements, uint ntrans, tfloat* d_weights, tfloat sigweight, tfloat sumweight,
                          tcomplex* d_output, tfloat* d_outputweights, tfloat* d_sigma2noise,
                          tfloat* d_normcorrection, tfloat* d_priorclass, tfloat* d_correctionxa,
                          tfloat* d_correctionaa, bool doscale) {
  check(gtomrln_store_weights_add(cf(d_input), d_ctf, cf(d_ref), d_minvsigma2, d_mresol, elements, ntrans,
                                  d_weights, sigweight, sumweight, f(d_output), d_outputweights, d_sigma2noise,
                                  d_normcorrection, d_priorclass, d_correctionxa, d_correctionaa, doscale, nullptr),
        "d_rlnStoreWeightsAdd");
}

// ------------------------------------------------------ RecFourier.cu ------
// include/Reconstruction.cuh:16, src/Reconstruction/RecFourier.cu:98-241
void d_ReconstructGridding(tcomplex* d_dataft, tfloat* d_weight, tfloat* d_reconstructed, int3 dimsori,
                           int3 dimspadded, int paddingfactor, cufftHandle pre_planforw, cufftHandle pre_planback,
                           int iterations, double blobradius, int bloborder, double blobalpha) {
  check(gtomrln_reconstruct_gridding(cf(d_dataft), d_weight, d_reconstructed, dimsori.x, dimsori.y, dimsori.z,
                                     dimspadded.x, dimspadded.y, dimspadded.z, paddingfactor, (int)pre_planforw,
                                     (int)pre_planback, iterations, blobradius, bloborder, blobalpha, nullptr),
        "d_ReconstructGridding");
}

}  // namespace gtom
