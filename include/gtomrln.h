/*
 * gtomrln.h — C ABI of the B200 RELION-style Fourier projector, backprojector
 * and gridding reconstructor.
 *
 * Every entry point is a drop-in for one overload of gtom's C++ API
 * (namespace gtom, include/Relion.cuh and include/Reconstruction.cuh of
 * dtegunov/gtom); the reference declaration it replaces is cited above each
 * one.  The arguments keep the reference's meaning and order; C types replace
 * the C++ ones:
 *
 *   tcomplex*      -> float*  interleaved (re, im) pairs, 8-byte aligned
 *   tfloat*        -> float*
 *   int3 dims      -> three ints (x, y, z); a 2D slice has z == 1
 *   glm::mat3*     -> float*  9 floats per matrix, column-major (glm layout)
 *   tfloat3* angles-> float*  3 floats per slice: rot, tilt, psi in radians
 *   float4 mag     -> four floats (the columns of the 2x2 magnification)
 *   cudaTex        -> unsigned long long (cudaTextureObject_t)
 *   cufftHandle    -> int (0 = let the library plan)
 *
 * One argument is added at the end of each call: a cudaStream_t passed as
 * void* (NULL = the legacy default stream).  The reference runs on the
 * default stream and returns only after its work is done; the entry points
 * here enqueue on the given stream and return once the work is enqueued, so
 * a caller that reads results on the host synchronises the stream first.
 *
 * Errors: every entry point returns GTOMRLN_OK (0) or a negative status and
 * never throws or terminates; gtomrln_last_error() returns the calling
 * thread's last message.  Where the reference calls `throw;` (which
 * terminates the process) on inconsistent dimensions, these return
 * GTOMRLN_ERR_INVALID.
 *
 * Memory: d_* pointers are caller-owned device buffers, h_* are caller-owned
 * host arrays read during the call.  Backprojection accumulates into
 * d_volumeft / d_volumeweights in place (the caller zeroes them first).
 */
#ifndef GTOMRLN_H
#define GTOMRLN_H

#if defined(__GNUC__)
#define GTOMRLN_API __attribute__((visibility("default")))
#else
#define GTOMRLN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GTOMRLN_OK 0
#define GTOMRLN_ERR_INVALID -1 /* inconsistent dimensions or arguments */
#define GTOMRLN_ERR_CUDA -2    /* a CUDA runtime call or launch failed */
#define GTOMRLN_ERR_CUFFT -3   /* cuFFT planning or execution failed */
#define GTOMRLN_ERR_ALLOC -4   /* device memory could not be allocated */

/* Library version (major * 10000 + minor * 100 + patch). */
GTOMRLN_API int gtomrln_version(void);

/* Message of the calling thread's last failed call ("" if none). */
GTOMRLN_API const char* gtomrln_last_error(void);

/* Release cached cuFFT plans and the library's memory pool on the current
 * device.  Not required; the caches are also released at process exit. */
GTOMRLN_API int gtomrln_release_caches(void);

/* Extension (no reference counterpart): choose the implementation of an
 * operation for the calling process.  op: GTOMRLN_OP_PROJECT or
 * GTOMRLN_OP_BACKPROJECT; path: GTOMRLN_PATH_AUTO (default: brick-major with
 * row segments for 2D slices whose geometry allows it, once the volume is
 * too large for L2 and the batch amortises the plan — backprojector: edge
 * >= 384 and >= 300 slices, or edge >= 256 and >= 6 000; projector: edge
 * >= 512 and >= 1 000, or edge >= 384 and >= 6 000 — else direct),
 * GTOMRLN_PATH_DIRECT (one thread per slice element, global gathers /
 * reductions), GTOMRLN_PATH_BRICK (brick-major, shared-memory staging, pixels
 * binned per brick by a planning pass; falls back to direct where the
 * geometry does not allow it) or GTOMRLN_PATH_SEGMENT (brick-major, pixels
 * found per brick by row segments instead of binning).  All paths compute
 * the same per-sample arithmetic. */
#define GTOMRLN_OP_PROJECT 0
#define GTOMRLN_OP_BACKPROJECT 1
/* op GTOMRLN_OP_GRIDDING: GTOMRLN_PATH_AUTO (default) runs the gridding
 * as GTOMRLN_PATH_SYMMETRIC (below) on the grids P = 64, 96, 128, 192, 256,
 * 512 and 800 and with cuFFT's 3D transforms elsewhere;
 * GTOMRLN_PATH_DIRECT always uses cuFFT; GTOMRLN_PATH_FUSED runs each
 * iteration as two fused passes with the library's own transforms on
 * power-of-two grids P = 64 .. 512 (cuFFT elsewhere). */
#define GTOMRLN_OP_GRIDDING 2
#define GTOMRLN_PATH_AUTO 0
#define GTOMRLN_PATH_DIRECT 1
#define GTOMRLN_PATH_BRICK 2
#define GTOMRLN_PATH_SEGMENT 3
#define GTOMRLN_PATH_FUSED 4
/* op GTOMRLN_OP_BACKPROJECT: the row-segment kernel with FP32 shared-memory
 * atomics only (GTOMRLN_PATH_SEGMENT and AUTO first accumulate each work
 * item in fixed point with int32 atomics, at the FP32 path's accuracy, and
 * fall back to FP32 for an item whose sums could overflow). */
#define GTOMRLN_PATH_SEGMENT_FP32 5
/* op GTOMRLN_OP_GRIDDING: each iteration as four streaming passes over the
 * Hermitian half along z of the (real) iterated spectrum, and the final map
 * as three passes that write only the cropped output, all with the library's
 * own transforms (no cuFFT plan), on the grids P = 64, 96, 128, 192, 256,
 * 512 and 800 (cuFFT elsewhere). */
#define GTOMRLN_PATH_SYMMETRIC 6
GTOMRLN_API int gtomrln_set_path(int op, int path);

/* Extension (no reference counterpart): launch shape of the brick-major
 * kernels of op for the calling process — brick edge in voxels, threads per
 * CTA (multiple of 32, <= 1024) and the most slices one work item takes.
 * 0 keeps the built-in default for that field.  Results do not depend on
 * these (the projector's are bit-identical for any shape); speed does.
 * Returns GTOMRLN_ERR_INVALID for shapes whose shared memory exceeds a CTA's. */
GTOMRLN_API int gtomrln_set_brick_tuning(int op, int edge, int threads, int chunk);

/* Host helper: M_b = transpose(Matrix3Euler(angles_b)) * supersample, the
 * matrices the h_angles overloads build (src/Relion/Project.cu:14-16,
 * src/Helpers/Euler.cu:39-68).  Writes 9 * batch floats, column-major. */
GTOMRLN_API int gtomrln_matrices_from_angles(const float* h_angles, float supersample, unsigned batch,
                                 float* h_matrices);

/* ---------------------------------------------------------------------------
 * Projector: trilinear central-slice gather from a decentred half-complex
 * volume of (dimsvolume.x/2+1) x dimsvolume.y x dimsvolume.z.  Output slices
 * are half-complex (dimsproj.x/2+1) x dimsproj.y [x dimsproj.z], one after
 * another; elements with x^2+y^2 > rmax^2 are written as 0.
 * ------------------------------------------------------------------------- */

/* gtom::d_rlnProject(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj,
 *     int3 dimsproj, uint rmax, glm::mat3* d_matrices, uint batch)
 * include/Relion.cuh:35, src/Relion/Project.cu:25-43 */
GTOMRLN_API int gtomrln_project(const float* d_volumeft, int vx, int vy, int vz, float* d_proj, int px,
                    int py, int pz, unsigned rmax, const float* d_matrices, unsigned batch,
                    void* stream);

/* gtom::d_rlnProject(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj,
 *     int3 dimsproj, tfloat3* h_angles, float supersample, uint batch)
 * include/Relion.cuh:34, src/Relion/Project.cu:12-23 (rmax = dimsproj.x/2) */
GTOMRLN_API int gtomrln_project_angles(const float* d_volumeft, int vx, int vy, int vz, float* d_proj,
                           int px, int py, int pz, const float* h_angles, float supersample,
                           unsigned batch, void* stream);

/* gtom::d_rlnProject(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume,
 *     tcomplex* d_proj, int3 dimsproj, uint rmax, glm::mat3* d_matrices, uint batch)
 * include/Relion.cuh:37, src/Relion/Project.cu:58-87.  The textures are read
 * at the same integer coordinates as the reference, so their filter and
 * address modes (set by the caller) act identically. */
GTOMRLN_API int gtomrln_project_tex(unsigned long long t_volumeRe, unsigned long long t_volumeIm, int vx,
                        int vy, int vz, float* d_proj, int px, int py, int pz, unsigned rmax,
                        const float* d_matrices, unsigned batch, void* stream);

/* Extension with no counterpart in the reference: gtomrln_project_angles
 * for callers that cannot allocate device memory — code whose device memory
 * is owned by another allocator (a host application's memory pool or a
 * fixed budget), or that must not let an allocation synchronise the device
 * in the middle of a pipeline.  The reference's h_angles overload, and
 * gtomrln_project_angles, place the rotation matrices in freshly allocated
 * device memory; this entry point uses a fixed array inside the library
 * instead and allocates nothing.  Limit: batch <= 4096 slices per call
 * (larger batches return GTOMRLN_ERR_INVALID; split them).  The array costs
 * every device that loads the library 147,456 bytes until the process exits.
 * Each call looks up the array's device address (on the first call on a
 * device this loads the library's device code); make the first call on a
 * device before any stream capture.  The matrices travel to the array as
 * kernel parameters, and the projection always runs the direct kernel (the
 * brick kernels would need plan scratch).  All calls share the one array,
 * which keeps the last call's matrices: calls ordered on one stream are
 * safe, calls on different streams that overlap on the GPU race.  Results
 * equal gtomrln_project_angles's. */
GTOMRLN_API int gtomrln_project_angles_noalloc(const float* d_volumeft, int vx, int vy, int vz,
                                   float* d_proj, int px, int py, int pz, const float* h_angles,
                                   float supersample, unsigned batch, void* stream);

/* gtom::d_rlnProject(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume,
 *     tcomplex* d_proj, int3 dimsproj, tfloat3* h_angles, float supersample, uint batch)
 * include/Relion.cuh:36, src/Relion/Project.cu:45-56 */
GTOMRLN_API int gtomrln_project_tex_angles(unsigned long long t_volumeRe, unsigned long long t_volumeIm,
                               int vx, int vy, int vz, float* d_proj, int px, int py, int pz,
                               const float* h_angles, float supersample, unsigned batch,
                               void* stream);

/* ---------------------------------------------------------------------------
 * Backprojector: trilinear scatter-insert of half-complex slices and their
 * per-pixel weights (CTF-weighted data and CTF^2, applied by the caller) into
 * a half-complex volume and a weight volume, accumulated in place.
 * d_projft == NULL inserts (1, 0); d_projweights == NULL inserts weight 1;
 * d_volumeft or d_volumeweights == NULL skips that output.  d_ivolume
 * (optional) selects a target volume per slice.  The trilinear weights are
 * rounded through binary16 exactly as the reference does
 * (src/Relion/Backproject.cu:224-238).
 * ------------------------------------------------------------------------- */

/* gtom::d_rlnBackproject(tcomplex* d_volumeft, tfloat* d_volumeweights,
 *     int3 dimsvolume, tcomplex* d_projft, tfloat* d_projweights, int3 dimsproj,
 *     uint rmax, glm::mat3* d_matrices, int* d_ivolume, float4 magnification,
 *     float ewaldradiussuper, bool outputdecentered, bool squareinterpweights,
 *     uint batch)
 * include/Relion.cuh:9, src/Relion/Backproject.cu:48-124 */
GTOMRLN_API int gtomrln_backproject(float* d_volumeft, float* d_volumeweights, int vx, int vy, int vz,
                        const float* d_projft, const float* d_projweights, int px, int py,
                        int pz, unsigned rmax, const float* d_matrices, const int* d_ivolume,
                        float mag_x, float mag_y, float mag_z, float mag_w,
                        float ewaldradiussuper, int outputdecentered, int squareinterpweights,
                        unsigned batch, void* stream);

/* gtom::d_rlnBackproject(tcomplex* d_volumeft, tfloat* d_volumeweights,
 *     int3 dimsvolume, tcomplex* d_projft, tfloat* d_projweights, int3 dimsproj,
 *     uint rmax, tfloat3* h_angles, int* h_ivolume, float4 magnification,
 *     float ewaldradius, float supersample, bool outputdecentered,
 *     bool squareinterpweights, uint batch)
 * include/Relion.cuh:10, src/Relion/Backproject.cu:23-46 */
GTOMRLN_API int gtomrln_backproject_angles(float* d_volumeft, float* d_volumeweights, int vx, int vy,
                               int vz, const float* d_projft, const float* d_projweights,
                               int px, int py, int pz, unsigned rmax, const float* h_angles,
                               const int* h_ivolume, float mag_x, float mag_y, float mag_z,
                               float mag_w, float ewaldradius, float supersample,
                               int outputdecentered, int squareinterpweights, unsigned batch,
                               void* stream);

/* gtom::d_BackprojectTomo(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_projft,
 *     tfloat* d_projweights, int3 dimsproj, uint rmax, glm::mat3* d_matrices, uint batch)
 * include/Relion.cuh:14, src/Relion/BackprojectTomo.cu:30-46, kernel :48-153: a gather
 * with a Lanczos-5 kernel instead of a scatter; every voxel of the decentred
 * half volume inside rmax with kernel weight sum above 1e-3 is overwritten
 * with sum(w v) / sum(w weight) times the clamped weight sum.  The volume
 * must be cubic; d_projweights is required (the reference reads it). */
GTOMRLN_API int gtomrln_backproject_tomo(float* d_volumeft, int vx, int vy, int vz, const float* d_projft,
                             const float* d_projweights, int px, int py, int pz, unsigned rmax,
                             const float* d_matrices, unsigned batch, void* stream);

/* gtom::d_BackprojectTomo(..., uint rmax, tfloat3* h_angles, uint batch)
 * include/Relion.cuh:13, src/Relion/BackprojectTomo.cu:11-28 (matrices
 * transpose(Euler), no supersampling). */
GTOMRLN_API int gtomrln_backproject_tomo_angles(float* d_volumeft, int vx, int vy, int vz,
                                    const float* d_projft, const float* d_projweights, int px,
                                    int py, int pz, unsigned rmax, const float* h_angles,
                                    unsigned batch, void* stream);

/* ---------------------------------------------------------------------------
 * Shifted projector / backprojector: the slices are multiplied by the phase
 * exp(-i (x sx + y sy [+ z sz])) of a per-slice shift and by a per-slice
 * global weight.  The matrix overloads take the shifts already scaled to
 * radians per pixel (pixels * 2 pi / dimsproj.x, float3 per slice) and the
 * weights in device memory; the h_angles overloads take pixels and scale
 * them.  The shifted backprojector is its own insertion in the reference
 * (no binary16 weights, no mirrored neighbours, the whole x = 0 column,
 * r^2 <= rmax^2, centred output) and is reproduced as such; the reference
 * writes without bounds checks, here indices are clamped as in
 * gtomrln_backproject.  NULL d_projft / d_projweights mean value 1 / weight 1.
 * ------------------------------------------------------------------------- */

/* gtom::d_rlnProjectShifted(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj,
 *     int3 dimsproj, uint rmax, glm::mat3* d_matrices, tfloat3* d_shifts,
 *     float* d_globalweights, uint batch)
 * include/Relion.cuh:41, src/Relion/ProjectShifted.cu:58-75, kernel :124-224. */
GTOMRLN_API int gtomrln_project_shifted(const float* d_volumeft, int vx, int vy, int vz, float* d_proj,
                            int px, int py, int pz, unsigned rmax, const float* d_matrices,
                            const float* d_shifts, const float* d_globalweights, unsigned batch,
                            void* stream);

/* gtom::d_rlnProjectShifted(tcomplex* d_volumeft, int3 dimsvolume, tcomplex* d_proj,
 *     int3 dimsproj, tfloat3* h_angles, tfloat3* h_shifts, float* h_globalweights,
 *     float supersample, uint batch)
 * include/Relion.cuh:40, src/Relion/ProjectShifted.cu:32-56 (rmax = dimsproj.x / 2). */
GTOMRLN_API int gtomrln_project_shifted_angles(const float* d_volumeft, int vx, int vy, int vz,
                                   float* d_proj, int px, int py, int pz, const float* h_angles,
                                   const float* h_shifts, const float* h_globalweights,
                                   float supersample, unsigned batch, void* stream);

/* gtom::d_rlnProjectShifted(cudaTex t_volumeRe, cudaTex t_volumeIm, int3 dimsvolume, ...,
 *     uint rmax, glm::mat3* d_matrices, tfloat3* d_shifts, float* d_globalweights, uint batch)
 * include/Relion.cuh:43, src/Relion/ProjectShifted.cu:103-122, kernel :226-338. */
GTOMRLN_API int gtomrln_project_shifted_tex(unsigned long long t_re, unsigned long long t_im, int vx,
                                int vy, int vz, float* d_proj, int px, int py, int pz,
                                unsigned rmax, const float* d_matrices, const float* d_shifts,
                                const float* d_globalweights, unsigned batch, void* stream);

/* gtom::d_rlnProjectShifted(cudaTex, cudaTex, int3, tcomplex*, int3, tfloat3* h_angles,
 *     tfloat3* h_shifts, float* h_globalweights, float supersample, uint batch)
 * include/Relion.cuh:42, src/Relion/ProjectShifted.cu:78-101. */
GTOMRLN_API int gtomrln_project_shifted_tex_angles(unsigned long long t_re, unsigned long long t_im,
                                       int vx, int vy, int vz, float* d_proj, int px, int py,
                                       int pz, const float* h_angles, const float* h_shifts,
                                       const float* h_globalweights, float supersample,
                                       unsigned batch, void* stream);

/* gtom::d_rlnBackprojectShifted(tcomplex* d_volumeft, tfloat* d_volumeweights,
 *     int3 dimsvolume, tcomplex* d_projft, tfloat* d_projweights, int3 dimsproj, uint rmax,
 *     glm::mat3* d_matrices, tfloat3* d_shifts, float* d_globalweights, uint batch)
 * include/Relion.cuh:18, src/Relion/BackprojectShifted.cu:37-58, kernel :60-186. */
GTOMRLN_API int gtomrln_backproject_shifted(float* d_volumeft, float* d_volumeweights, int vx, int vy,
                                int vz, const float* d_projft, const float* d_projweights,
                                int px, int py, int pz, unsigned rmax, const float* d_matrices,
                                const float* d_shifts, const float* d_globalweights,
                                unsigned batch, void* stream);

/* gtom::d_rlnBackprojectShifted(..., uint rmax, tfloat3* h_angles, tfloat3* h_shifts,
 *     float* h_globalweights, float supersample, uint batch)
 * include/Relion.cuh:17, src/Relion/BackprojectShifted.cu:11-35. */
GTOMRLN_API int gtomrln_backproject_shifted_angles(float* d_volumeft, float* d_volumeweights, int vx,
                                       int vy, int vz, const float* d_projft,
                                       const float* d_projweights, int px, int py, int pz,
                                       unsigned rmax, const float* h_angles,
                                       const float* h_shifts, const float* h_globalweights,
                                       float supersample, unsigned batch, void* stream);

/* ---------------------------------------------------------------------------
 * Gridding reconstructor: RELION-style iterative gridding-weight correction
 * with a Kaiser-Bessel blob, then the inverse FFT, crop and sinc^2 correction.
 * d_dataft / d_weight are CENTRED half-complex volumes of dimspadded (the
 * output of a centred backprojection); the working grid is
 * P = dimsori.x * paddingfactor.  d_reconstructed receives the real ori^3
 * map, centred.  Inputs are not modified.  dimspadded.x must be at least
 * P + 1: with a smaller box the reference reads outside its input (its
 * DecenterKernel, RecFourier.cu:264-285); here such reads are not made and
 * the masked values they would feed count as 0.
 * ------------------------------------------------------------------------- */

/* gtom::d_ReconstructGridding(tcomplex* d_dataft, tfloat* d_weight,
 *     tfloat* d_reconstructed, int3 dimsori, int3 dimspadded, int paddingfactor = 2,
 *     cufftHandle pre_planforw = NULL, cufftHandle pre_planback = NULL,
 *     int iterations = 10, double blobradius = 1.9, int bloborder = 0,
 *     double blobalpha = 15)
 * include/Reconstruction.cuh:16, src/Reconstruction/RecFourier.cu:98-241.
 * pre_planforw / pre_planback: 0 lets the library use its own cached plans
 * for the P^3 R2C / C2R transforms; otherwise they must be such plans.  They
 * are used only where the gridding runs on cuFFT (GTOMRLN_PATH_DIRECT, or a
 * grid the library's own transforms do not take). */
GTOMRLN_API int gtomrln_reconstruct_gridding(const float* d_dataft, const float* d_weight,
                                 float* d_reconstructed, int ox, int oy, int oz, int padx,
                                 int pady, int padz, int paddingfactor, int pre_planforw,
                                 int pre_planback, int iterations, double blobradius,
                                 int bloborder, double blobalpha, void* stream);

/* Extension (no reference counterpart): the same reconstruction with a
 * convergence test.  Iterates at most max_iterations times and stops early
 * once the relative L2 change of the corrected weights Fweight * Fnewweight
 * between two iterations, ||Fw (Fnw' - Fnw)|| / ||Fw Fnw||, is <= tolerance
 * (voxels that received no weight do not count; their Fnewweight only grows
 * towards the 1e20 clamp).  tolerance <= 0 disables the test, which then
 * equals gtomrln_reconstruct_gridding).  *iterations_done and
 * *final_change (either may be NULL) receive the count and the last
 * relative change.  Synchronises the stream once per iteration. */
GTOMRLN_API int gtomrln_reconstruct_gridding_tol(const float* d_dataft, const float* d_weight,
                                     float* d_reconstructed, int ox, int oy, int oz, int padx,
                                     int pady, int padz, int paddingfactor, int max_iterations,
                                     double tolerance, double blobradius, int bloborder,
                                     double blobalpha, int* iterations_done,
                                     double* final_change, void* stream);

/* Extension (no reference counterpart): the gridding reconstruction with a
 * learned warm start and/or momentum.
 *   d_mlp_params: NULL for the reference's sphere-mask start, else the
 *     parameter block of the per-voxel MLP (gtomrln_mlp_param_count()
 *     floats, device memory; layout in gtom_b200/csrc/mlp.cuh), which
 *     predicts the converged Fnewweight from the 27 log-weights around each
 *     voxel and its radius.  The first iteration from the predicted start is
 *     its residual check: if its relative change exceeds residual_limit (or
 *     is not finite) the prediction is discarded and the iteration restarts
 *     from the sphere mask (*warm_used = 0; the rejected iteration still
 *     counts in *iterations_done).
 *   momentum: 0 for the reference's update Fnw <- Fnw / max(1e-4, c); in
 *     (0, 1) the update is applied at the extrapolated point
 *     V = Fnw' (Fnw' / Fnw)^momentum (same fixed points, far fewer
 *     iterations to a given distance from them).
 * max_iterations / tolerance / *iterations_done / *final_change as in
 * gtomrln_reconstruct_gridding_tol; any output pointer may be NULL. */
GTOMRLN_API int gtomrln_reconstruct_gridding_warm(const float* d_dataft, const float* d_weight,
                                      float* d_reconstructed, int ox, int oy, int oz, int padx,
                                      int pady, int padz, int paddingfactor, int max_iterations,
                                      double tolerance, float momentum,
                                      const float* d_mlp_params, float residual_limit,
                                      double blobradius, int bloborder, double blobalpha,
                                      int* iterations_done, double* final_change, int* warm_used,
                                      void* stream);

/* Extension (no reference counterpart): only the gridding weights of
 * gtomrln_reconstruct_gridding_warm for the weights d_weight (centred half
 * volume of dims ox x oy x oz, at least P + 1 with P = ori * paddingfactor):
 * d_fnw receives Fnewweight and d_fw (may be NULL) the decentred, masked
 * Fweight, both on the decentred (P/2+1) x P x P grid.  Used to make the
 * MLP's training pairs and to compare starts.  d_ref_fnw (may be NULL):
 * reference weights on the same grid, e.g. converged ones; each iteration
 * then measures the distance ||Fw (Fnw - ref)|| / ||Fw ref|| and the loop
 * also stops once it is <= ref_tolerance (*final_distance receives the
 * last one; the cuFFT path runs whatever path is selected). */
GTOMRLN_API int gtomrln_gridding_weights(const float* d_weight, int ox, int oy, int oz, int ori,
                             int paddingfactor, int max_iterations, double tolerance,
                             float momentum, const float* d_mlp_params, float residual_limit,
                             double blobradius, int bloborder, double blobalpha, float* d_fw,
                             float* d_fnw, int* iterations_done, double* final_change,
                             int* warm_used, const float* d_ref_fnw, double ref_tolerance,
                             double* final_distance, void* stream);

/* ---------------------------------------------------------------------------
 * The warm-start MLP (no reference counterpart).  28 inputs -> 64 -> 64 -> 1,
 * ReLU, FP32; parameters, gradients and Adam moments are arrays of
 * gtomrln_mlp_param_count() floats with the layout of
 * gtom_b200/csrc/mlp.cuh (the first 56 entries, the input standardisation,
 * are not trained).  Features are the raw 28 inputs of a voxel (27
 * log-weights, radius); targets are log(Fnewweight * s).
 * ------------------------------------------------------------------------- */
GTOMRLN_API int gtomrln_mlp_param_count(void);

/* d_out[i] = network output for the raw features d_features[i*28 .. +28). */
GTOMRLN_API int gtomrln_mlp_forward(const float* d_params, const float* d_features, int n,
                        float* d_out, void* stream);

/* Raw features of n voxels of a stack of decentred half grids of P (each
 * (P/2+1) x P x P floats of Fweight): voxel i is element d_index[i] of the
 * stack, whose volume v = d_index[i] / ((P/2+1) P P) has weight scale
 * 1 / d_inv_scale[v]. */
GTOMRLN_API int gtomrln_mlp_volume_features(const float* d_fw, int P, const float* d_inv_scale,
                                const long long* d_index, int n, float* d_features,
                                void* stream);

/* Loss L = loss_scale * sum_i w_i (out_i - t_i)^2 over n samples given as
 * raw features, added to *d_loss; dL/dparams added to d_grad. */
GTOMRLN_API int gtomrln_mlp_gradients(const float* d_params, const float* d_features,
                          const float* d_targets, const float* d_weights, int n,
                          float loss_scale, float* d_grad, float* d_loss, void* stream);

/* The same for samples gathered from a stack of half grids (as in
 * gtomrln_mlp_volume_features); d_target / d_weight are stacks of the same
 * shape holding each voxel's target and loss weight. */
GTOMRLN_API int gtomrln_mlp_train_batch(const float* d_params, const float* d_fw,
                            const float* d_target, const float* d_weight,
                            const float* d_inv_scale, int P, const long long* d_index, int n,
                            float loss_scale, float* d_grad, float* d_loss, void* stream);

/* One Adam step (step counts from 1) on the trained entries; zeroes d_grad. */
GTOMRLN_API int gtomrln_mlp_adam(float* d_params, float* d_grad, float* d_m, float* d_v, int step,
                     float lr, float beta1, float beta2, float eps, void* stream);

/* ---------------------------------------------------------------------------
 * CTF and particle preprocessing (the step before insertion).
 * ------------------------------------------------------------------------- */

/* gtom::CTFParams (include/CTF.cuh:11-42): lengths in metres, angles in
 * radians; the reference's defaults are pixelsize 1e-10, Cs 2e-3, voltage
 * 300e3, defocus -3e-6, amplitude 0.07, scale 1, all else 0. */
typedef struct gtomrln_ctf_params {
  float pixelsize, pixeldelta, pixelangle, Cs, voltage, defocus, astigmatismangle, defocusdelta,
      amplitude, Bfactor, Bfactordelta, Bfactorangle, scale, phaseshift;
} gtomrln_ctf_params_t;

/* gtom::d_CTFSimulate(CTFParams* h_params, float2* d_addresses, float* d_gammacorrection,
 *     tfloat* d_output, uint n, bool amplitudesquared = false, bool ignorefirstpeak = false,
 *     int batch = 1)
 * include/CTF.cuh:317, src/CTF/Simulate.cu:22-47, kernel :117-139, d_GetCTF
 * include/CTF.cuh:195-223.  d_addresses: n float2 (spatial frequency in
 * 1/pixel, azimuth); d_gammacorrection may be NULL; d_output: batch x n. */
GTOMRLN_API int gtomrln_ctf_simulate(const gtomrln_ctf_params_t* h_params, const float* d_addresses,
                         const float* d_gammacorrection, float* d_output, unsigned n,
                         int amplitudesquared, int ignorefirstpeak, int batch, void* stream);

/* Extension (no single reference function; the steps a caller of
 * d_rlnBackproject makes before it): batch real-space particles of n x n
 * (row-major, centred at (n/2, n/2)) to d_projft = CTF * FT and
 * d_projweights = CTF^2 (may be NULL), both half-complex (n/2+1) x n per
 * particle, ready for gtomrln_backproject.  FT is cuFFT's unnormalised R2C
 * of the particle moved to the origin (a factor (-1)^(x+y)); the CTF at
 * each element is gtomrln_ctf_simulate's for the address
 * (sqrt(x^2 + y^2) / n, atan2(y, x)).  h_params NULL: no CTF (weights 1).
 * batch <= 65535. */
GTOMRLN_API int gtomrln_preprocess_particles(const float* d_images, int n, unsigned batch,
                                 const gtomrln_ctf_params_t* h_params, float* d_projft,
                                 float* d_projweights, void* stream);

/* ---------------------------------------------------------------------------
 * RELION E-step consumers of the projections.  Complex arrays are
 * interleaved float pairs; uint3 / uint4 arrays are 3 / 4 unsigned per item.
 * ------------------------------------------------------------------------- */

/* gtom::d_rlnSquaredDifferencesSparse(tcomplex* d_particleft, tfloat* d_minvsigma2,
 *     tfloat* d_ctf, int3 dimsparticle, tcomplex* d_precalcshifts, tcomplex* d_refft,
 *     tfloat* d_diff2, uint3* d_combination, uint ncombinations, uint groupsize,
 *     bool dofirstitercc)
 * include/Relion.cuh:48; the reference declares it but src/Relion/SquaredDifferences.cu
 * is empty: defined here from GTOMTest/RelionSquaredDiff.cpp:55-69.  Combination k
 * = (first shift, particle, first reference) covers groupsize x groupsize outputs
 * d_diff2[k g^2 + r g + s] = 0.5 sum_i minvsigma2_i |ctf_i ref_{z+r,i} - part_i shift_{x+s,i}|^2
 * (ctf of the particle y, elements per particle; NULL minvsigma2 / ctf = 1), or
 * with dofirstitercc the negative cross-correlation normalised by the
 * reference power.  ncombinations counts outputs; groupsize 1, 2, 4 or 8. */
GTOMRLN_API int gtomrln_squared_differences_sparse(const float* d_particleft, const float* d_minvsigma2,
                                       const float* d_ctf, int dx, int dy, int dz,
                                       const float* d_precalcshifts, const float* d_refft,
                                       float* d_diff2, const unsigned* d_combination,
                                       unsigned ncombinations, unsigned groupsize,
                                       int dofirstitercc, void* stream);

/* gtom::d_rlnSquaredDifferences (include/Relion.cuh:46; no reference source,
 * see above): every particle against every reference and shift,
 * d_diff2[(particle * nrefs + ref) * nshifts + shift], tile 1, 2, 4 or 8. */
GTOMRLN_API int gtomrln_squared_differences(const float* d_particleft, const float* d_minvsigma2,
                                const float* d_ctf, int dx, int dy, int dz, unsigned nparticles,
                                const float* d_precalcshifts, unsigned nshifts,
                                const float* d_refft, unsigned nrefs, unsigned tile,
                                float* d_diff2, int dofirstitercc, void* stream);

/* gtom::d_rlnConvertWeightsDense — include/Relion.cuh:21, src/Relion/ConvertWeights.cu:12-44. */
GTOMRLN_API int gtomrln_convert_weights_dense(float* d_weights, unsigned nparticles, unsigned nclasses,
                                  unsigned nrot, unsigned ntrans, const float* d_pdfrot,
                                  const float* d_pdftrans, const float* d_mindiff2, void* stream);

/* gtom::d_rlnConvertWeightsSparse — include/Relion.cuh:22, ConvertWeights.cu:46-73. */
GTOMRLN_API int gtomrln_convert_weights_sparse(float* d_weightsdense, float* d_weightssparse,
                                   const unsigned* d_combinations, unsigned nsparse, unsigned nrot,
                                   unsigned ntrans, const float* d_pdfrot, const float* d_pdftrans,
                                   const float* d_mindiff2, void* stream);

/* gtom::d_rlnConvertWeightsSort (ascending, in place) — include/Relion.cuh:23,
 * ConvertWeights.cu:75-78. */
GTOMRLN_API int gtomrln_convert_weights_sort(float* d_input, unsigned n, void* stream);

/* gtom::d_rlnConvertWeightsCompact (the positive values, in order; *n in:
 * input length, out: kept count; synchronises the stream) —
 * include/Relion.cuh:24, ConvertWeights.cu:80-91. */
GTOMRLN_API int gtomrln_convert_weights_compact(const float* d_input, float* d_output, unsigned* n,
                                    void* stream);

/* gtom::d_rlnDiffRemapDense — include/Relion.cuh:27, src/Relion/DiffRemap.cu:9-18, :30-51. */
GTOMRLN_API int gtomrln_diff_remap_dense(const float* d_input, float* d_output,
                             const unsigned* d_orientationindices, unsigned norientations,
                             unsigned iclass, unsigned nparticles, unsigned nclasses, unsigned nrot,
                             unsigned ntrans, unsigned ntranspadded, const float* d_xi2imgs,
                             const float* d_sqrtxi2, int docc, void* stream);

/* gtom::d_rlnDiffRemapSparse — include/Relion.cuh:28, DiffRemap.cu:20-28, :65-88
 * (d_mindiff2 receives the per-particle minimum, min-combined with its contents;
 * no limit on the particle count). */
GTOMRLN_API int gtomrln_diff_remap_sparse(const float* d_input, float* d_output, float* d_mindiff2,
                              const unsigned* d_combinations, const unsigned* d_hiddenover,
                              unsigned elements, unsigned tileelements, unsigned weightsperpart,
                              unsigned nparticles, const float* d_xi2imgs, const float* d_sqrtxi2,
                              int docc, void* stream);

/* gtom::d_rlnCreateMinvsigma2s — include/Relion.cuh:31, src/Relion/Misc.cu:12-29. */
GTOMRLN_API int gtomrln_create_minvsigma2s(float* d_output, const int* d_mresol, unsigned elements,
                               const float* d_sigma2noise, float sigma2fudge, void* stream);

/* gtom::d_rlnStoreWeightsAdd — include/Relion.cuh:51-57, src/Relion/StoreWeights.cu:9-63. */
GTOMRLN_API int gtomrln_store_weights_add(const float* d_input, const float* d_ctf, const float* d_ref,
                              const float* d_minvsigma2, const int* d_mresol, unsigned elements,
                              unsigned ntrans, const float* d_weights, float sigweight,
                              float sumweight, float* d_output, float* d_outputweights,
                              float* d_sigma2noise, float* d_normcorrection,
                              const float* d_priorclass, float* d_correctionxa,
                              float* d_correctionaa, int doscale, void* stream);

/* ---------------------------------------------------------------------------
 * Batched reconstruction of many volumes of uneven box size (no reference
 * counterpart; the reference batches equal boxes only, through d_ivolume of
 * d_rlnBackproject, src/Relion/Backproject.cu:48-124).  Per subvolume the
 * result equals gtomrln_backproject (matrix overload, rmax = box / 2,
 * identity magnification, flat Ewald sphere, centred accumulators of
 * dims P + 1, P = box * paddingfactor, zeroed first) followed by
 * gtomrln_reconstruct_gridding (ori = box, dimspadded = P + 1, the given
 * iteration count, blob radius 1.9, order 0, alpha 15): up to the order of
 * the floating-point additions of the insertion.
 * ------------------------------------------------------------------------- */
typedef struct gtomrln_subvolume {
  int box;                     /* even, >= 4 */
  int nslices;                 /* 2D slices of box x box, half-complex */
  const float* d_projft;       /* nslices x (box/2+1) x box complex64, or NULL (value 1) */
  const float* d_projweights;  /* nslices x (box/2+1) x box float, or NULL (weight 1) */
  const float* d_matrices;     /* nslices x 9 floats, as gtomrln_backproject's */
  float* d_out;                /* box^3 floats: the reconstructed map */
} gtomrln_subvolume_t;

/* Plans a batch: groups the subvolumes by box size, allocates the
 * accumulators and the gridding buffers of every size class (device memory
 * held until gtomrln_batch_destroy) and makes the batched FFT plans.  The
 * device pointers in items must stay valid for the handle's life; their
 * contents are read at each run. */
GTOMRLN_API int gtomrln_batch_create(const gtomrln_subvolume_t* items, int count, int paddingfactor,
                         int iterations, void** handle);

/* Launch shape of the persistent insertion kernel: threads per CTA
 * (multiple of 32, <= 1024), slices per work item, CTAs per SM; 0 keeps a
 * field.  Discards a captured graph. */
GTOMRLN_API int gtomrln_batch_set_tuning(void* handle, int threads, int slices_per_item,
                             int blocks_per_sm);

/* Runs the batch on stream: zeroes the accumulators, inserts every slice of
 * every subvolume in one persistent launch, then grids each size class.
 * use_graph != 0: the first call captures the sequence into a CUDA graph
 * (on a stream of the handle's own) and every call launches that graph on
 * `stream`; use_graph = 0 enqueues the steps directly.  Asynchronous. */
GTOMRLN_API int gtomrln_batch_run(void* handle, int use_graph, void* stream);

GTOMRLN_API int gtomrln_batch_destroy(void* handle);

/* The normalised Kaiser-Bessel table the gridding uses: nsamples values of
 * kaiser_Fourier_value(i * 0.5 / nsamples, radius, alpha, order) divided by
 * the value at 0 (src/Helpers/KaiserBessel.cpp:357-376,
 * src/Reconstruction/RecFourier.cu:104-116).  order must be 0 or 2. */
GTOMRLN_API int gtomrln_kaiser_bessel_table(double radius, double alpha, int order, int nsamples,
                                float* h_out);

#ifdef __cplusplus
}
#endif

#endif /* GTOMRLN_H */
