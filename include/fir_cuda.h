/*
 * fir_cuda.h -- C ABI of the B200 (sm_100a) implementation of FIR's
 * projection and reconstruction path.
 *
 * This is the drop-in boundary.  It replaces, call for call, the C++ entry
 * points of FIR's L4 layer (paths inside the FIR project):
 *
 *   fir_forward            projections::forward            src_lib/projections.h:9-12, projections.cc:15-92
 *   fir_backward           projections::backward           src_lib/projections.h:14-18, projections.cc:94-184
 *   fir_sensitivity        projections::computeSensitivityVol  src_lib/projections.h:20-24, projections.cc:186-197
 *   fir_osem_subiteration  one sub-iteration of reconAlgos::OSEM  src_lib/reconAlgos.cc:119-198
 *   fir_osem               reconAlgos::OSEM                src_lib/reconAlgos.h:29-36, reconAlgos.cc:63-201
 *   fir_ratio_backprojection  the getLine/ratio/projectLineIntegral loop of OSEM and OSEM_ResoReco  src_lib/reconAlgos.cc:119-158, :273-312
 *   fir_osem_psf              reconAlgos::OSEM_ResoReco, corrected (PSF in the model)              src_lib/reconAlgos.cc:203-367
 *   fir_osem_reso_reco        reconAlgos::OSEM_ResoReco as FIR runs it                           src_lib/reconAlgos.h:38-45, reconAlgos.cc:203-367
 *   fir_convolve           operations::convolve            src_lib/operations.h:7-10, operations.cc:11-192
 *   fir_cut_circle         operations::cutCircle           src_lib/operations.h:13-15, operations.cc:194-220
 *   fir_apply_mask         operations::applyMask           src_lib/operations.h:19, operations.cc:222-241
 *   fir_hu_to_mu           operations::HounsfieldToMuMap   src_lib/operations.h:22, operations.cc:243-284
 *   fir_proj_exponential   ProjData::exponential           src_lib/ProjData.h:108, ProjData.cc:514-539
 *   fir_proj_multiply      ProjData::operator*=            src_lib/ProjData.h:107, ProjData.cc:481-512
 *   fir_bin_coordinates    ProjData::getBinCoordinates     src_lib/ProjData.h:96-104, ProjData.cc:342-479
 *   fir_proj_rebin_weight  ProjData::rebinWeight           src_lib/ProjData.h:112, ProjData.cc:541-615
 *   fir_em_update          VolData /=, *= of the EM update src_lib/VolData.cc:305-343, reconAlgos.cc:161-166
 *   fir_lor_paths          Siddon::computePathBetweenCrystals (path dump) src_lib/Siddon.cc:88-258
 *   fir_siddon_paths       Siddon::computePath (path dump) src_lib/Siddon.h:45-55
 *   fir_proj_geometry      ProjHeader::check + ProjGeometry::fill  src_lib/ProjHeader.cc:6-186
 *   fir_scanner_tables     ScannerHeader::check + ScannerData position tables  src_lib/ScannerHeader.cc:26-342, ScannerData.cc:248-377
 *
 * Conventions
 *   - Every entry point returns a fir_status; FIR_OK is 0.  On failure
 *     fir_last_error() returns the message (thread-local), worded as FIR's
 *     own error() text where FIR has one.  No entry point throws.
 *   - Data pointers may be device pointers (work is enqueued on the context's
 *     stream and the call returns without waiting) or host pointers (the
 *     library stages them through device memory it owns, and the call
 *     returns when the results are back in host memory).
 *   - Sinograms are float32, segments -segOffset..+segOffset concatenated,
 *     each [view][axial][tang] (FIR's file order, ProjInterfileReader.cc:78-93).
 *     Volumes are float32 [frame][z][y][x] (VolData.h:151-156).
 *   - One context per host thread or stream; calls on different contexts
 *     may run concurrently.  A context is not thread-safe.
 */
#ifndef FIR_CUDA_H
#define FIR_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; these entry points are its
 * exported interface. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define FIR_CUDA_ABI_VERSION 1

typedef enum fir_status
{
  FIR_OK = 0,
  FIR_ERR_INVALID_ARGUMENT = 1, /* header or parameter rejected (FIR's error()) */
  FIR_ERR_CUDA = 2,             /* a CUDA runtime call failed */
  FIR_ERR_OUT_OF_MEMORY = 3,
  FIR_ERR_DEVICE_CHECK = 4,     /* a device-side check tripped (see message) */
  FIR_ERR_NO_DEVICE = 5,
  FIR_ERR_NOT_SUPPORTED = 6
} fir_status;

/* VolHeader (src_lib/VolHeader.h:7-23).  offset_x/y: centre of the first
 * voxel; offset_z: z offset of the volume centre from the scanner centre. */
typedef struct fir_vol_desc
{
  int nx, ny, nz;
  double voxel_x, voxel_y, voxel_z;
  double offset_x, offset_y, offset_z;
  int n_frames;
} fir_vol_desc;

/* ProjHeader (src_lib/ProjHeader.h:15-40).  n_tang_coords = 0 selects the
 * maximum, n_crystals_per_ring - 1. */
typedef struct fir_proj_desc
{
  int n_rings;
  int n_crystals_per_ring;
  int segment_span;
  int n_segments;
  int n_tang_coords;
} fir_proj_desc;

/* ProjGeometry (src_lib/ProjHeader.h:42-80); n_axial is returned separately. */
typedef struct fir_proj_info
{
  long long n_bins;
  int seg_offset;
  int tang_offset;
  int n_views;
  int half_span;
  int max_ring_diff;
  int n_tang_coords;
} fir_proj_info;

/* ScannerHeader (src_lib/ScannerHeader.h:7-46); zero dimensions mean "fit
 * tightly on the level below". */
typedef struct fir_scanner_desc
{
  double crystal_dims[3];
  int crystal_repeat[2];
  double inter_crystal[2];
  double module_dims[3];
  int module_repeat[2];
  double inter_module[2];
  double rsector_dims[3];
  int rsector_repeat;
  double rsector_inner_radius;
} fir_scanner_desc;

/* OSEMCoreParams (src_lib/reconAlgos.h:9-22). */
typedef struct fir_osem_params
{
  int n_iterations;
  int n_subsets;
  int save_interval;
  float cut_radius;
  int convolution_interval;
  float fwhm_xyz[3];
} fir_osem_params;

typedef struct fir_ctx fir_ctx;

/* Context options (fir_ctx_set_option). */
typedef enum fir_option
{
  /* FIR_GEOMETRY_REFERENCE (default): voxel extents are truncated to whole
   * millimetres for the traversal, exactly as FIR stores them in int
   * (Siddon.h:15-16,113).  FIR_GEOMETRY_EXACT: real-valued extents.  The two
   * agree for integer voxel sizes. */
  FIR_OPT_GEOMETRY = 1,
  /* FIR_BACKPROJ_ATOMIC (default): float atomics, order-nondeterministic
   * like FIR's "omp atomic".  FIR_BACKPROJ_DETERMINISTIC: contributions are
   * sorted per voxel into FIR's serial LOR order and summed in that order
   * with FIR's rounding, reproducing a single-threaded FIR run. */
  FIR_OPT_BACKPROJ_MODE = 2,
  /* 1: skip sinogram bins whose value is exactly 0 in backprojection and
   * OSEM (their contribution is exactly 0).  Default 0.  In the atomic mode
   * the OSEM sub-iteration and fir_backward first list a subset's non-zero
   * bins on the device (5 bytes of context scratch per LOR of the subset)
   * and trace only those; the result equals the full enumeration's up to the
   * order of the float atomic additions. */
  FIR_OPT_SKIP_ZERO_BINS = 3,
  /* Threads per block of the projector kernels (32..256, multiple of 32);
   * 0 restores the default. */
  FIR_OPT_BLOCK_SIZE = 4,
  /* 1: bracket every projector-kernel launch (forward, backward,
   * sensitivity, OSEM sub-iteration) with CUDA events on the context's
   * stream; read the accumulated device time with fir_ctx_projector_time. */
  FIR_OPT_TIMING = 5,
  /* Deterministic backprojection works on chunks of at most this many
   * (voxel, contribution) pairs (12 bytes each, twice, plus sort space);
   * 0 restores the default of 2^28.  Any chunk size gives the same result. */
  FIR_OPT_DETERMINISTIC_CHUNK = 6,
  /* Testing aid for failure reporting.  k > 0 bounds every traversal at k
   * steps and evaluates FIR's tie test as written (no fast form); a traversal
   * that reaches the bound before its end sets the device check word, and
   * the call reports FIR_ERR_DEVICE_CHECK (host buffers) or the next
   * fir_ctx_synchronize does.  Results past the bound are truncated.  0
   * (default): the natural bound, which only non-finite input can reach. */
  FIR_OPT_STEP_LIMIT = 7,
  /* FIR_TRAVERSAL_EXACT (default): FIR's double-precision traversal, voxel
   * lists and lengths bit-identical to FIR's.  FIR_TRAVERSAL_FLOAT (opt-in,
   * no counterpart in FIR): FIR's double set-up, then the loop in float with
   * float accumulation, for the OSEM sub-iteration's projection and
   * backprojection (fir_osem_subiteration, fir_osem, fir_ratio_backprojection
   * in the atomic backprojection mode).  It changes the voxel lists of a few
   * per cent of LORs (2.9 % of the clinical workload's) and line integrals by
   * up to about 1 %; OSEM images stay within 1e-4 relative L2 of the exact
   * mode's on the tested workloads.  The other projectors stay exact. */
  FIR_OPT_TRAVERSAL = 8
} fir_option;

enum
{
  FIR_GEOMETRY_REFERENCE = 0,
  FIR_GEOMETRY_EXACT = 1,
  FIR_BACKPROJ_ATOMIC = 0,
  FIR_BACKPROJ_DETERMINISTIC = 1,
  FIR_TRAVERSAL_EXACT = 0,
  FIR_TRAVERSAL_FLOAT = 1
};

/* ---- library / host helpers (no GPU needed) ---- */
int fir_abi_version(void);
const char* fir_last_error(void);
const char* fir_status_string(fir_status s);

/* ProjHeader::check + ProjGeometry::fill.  desc->n_tang_coords = 0 is
 * resolved in *geom.  n_axial: optional, room for desc->n_segments ints. */
fir_status fir_proj_geometry(const fir_proj_desc* desc, fir_proj_info* geom, int* n_axial);

/* ScannerHeader::check + ScannerData tables.  xy: 2*n_crystals_per_ring
 * doubles (x,y interleaved); z: 2*n_rings-1 doubles (slice centres).  Either
 * may be NULL to query n_rings / n_crystals_per_ring only. */
fir_status fir_scanner_tables(const fir_scanner_desc* desc, double* xy, double* z, int* n_rings,
                              int* n_crystals_per_ring);

/* ---- contexts ---- */
fir_status fir_ctx_create(fir_ctx** ctx, int device);
fir_status fir_ctx_destroy(fir_ctx* ctx);
/* stream: a cudaStream_t (NULL = legacy default stream). */
fir_status fir_ctx_set_stream(fir_ctx* ctx, void* stream);
fir_status fir_ctx_set_option(fir_ctx* ctx, fir_option opt, int value);
fir_status fir_ctx_get_option(fir_ctx* ctx, fir_option opt, int* value);
/* Uploads the scanner's crystal and slice position tables. */
fir_status fir_ctx_set_scanner(fir_ctx* ctx, const fir_scanner_desc* scanner);
/* Waits for the context's stream and reports device-side check failures. */
fir_status fir_ctx_synchronize(fir_ctx* ctx);
/* Number of kernels this context launched since creation (all entry points). */
long long fir_ctx_launch_count(const fir_ctx* ctx);
/* With FIR_OPT_TIMING on: waits for the recorded events and returns the total
 * device time (ms) and number of projector-kernel launches since the last
 * reset; reset != 0 clears the totals. */
fir_status fir_ctx_projector_time(fir_ctx* ctx, double* ms, long long* launches, int reset);

/* ---- projectors ---- */
/* projections::forward: sino[b] = sum over the Siddon path of bin b of
 * length * img, img being frame 0 of vol (VolData active frame 0). */
fir_status fir_forward(fir_ctx* ctx, const fir_vol_desc* vol, const float* img,
                       const fir_proj_desc* proj, float* sino);

/* Forward projection of an attenuation map followed by FIR's
 * ProjData::exponential in the same kernel: acf[b] = exp(line) if line >
 * 1e-5, else 1 (the attenuation correction factors of src_bin/OSEM.cc:294-311,
 * without the HU conversion). */
fir_status fir_forward_exp(fir_ctx* ctx, const fir_vol_desc* vol, const float* mu,
                           const fir_proj_desc* proj, float* acf);

/* projections::backward: img (n_subsets frames) is zeroed, then the bins of
 * subset s (views v with v % n_subsets == s) are backprojected into frame s. */
fir_status fir_backward(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino,
                        const fir_vol_desc* vol, float* img, int n_subsets);

/* projections::computeSensitivityVol: backward of an all-ones sinogram. */
fir_status fir_sensitivity(fir_ctx* ctx, const fir_proj_desc* proj, const fir_vol_desc* vol,
                           float* sens, int n_subsets);

/* ---- OSEM ---- */
/* One sub-iteration of reconAlgos::OSEM (reconAlgos.cc:119-187): for every
 * bin of subset `subset`, line = projection of img (+ bias), and if line >
 * 1e-5 the ratio sino/line is backprojected; then img *= bp / sens_frame
 * with FIR's 1e-5 gates, then the Gaussian filter if subiter %
 * convolution_interval == 0, then the cylindrical cut.  subiter is the
 * 1-based sub-iteration number.  bias may be NULL. */
fir_status fir_osem_subiteration(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino,
                                 const float* bias, const fir_vol_desc* vol, float* img,
                                 const float* sens_frame, const fir_osem_params* params,
                                 int subset, int subiter);

/* The same OSEM sub-iteration for callers that cannot allocate GPU memory
 * once they are running: reconstruction services that reserve their whole
 * device-memory budget at start-up and forbid later allocations (an
 * allocation can fail or stall when the budget is spent or fragmented), and
 * hosts whose GPU memory belongs to their own pool allocator, where an
 * allocation by the library would fail or force the pool to give memory
 * back.  This entry point has no counterpart in FIR.
 *
 * It allocates nothing and needs no context: every pointer (sinogram, bias,
 * image, sensitivity frame, and the scanner tables crystal_xy = 2 *
 * n_crystals_per_ring doubles and slice_z = 2 * n_rings - 1 doubles, as
 * fir_scanner_tables returns them) must be device memory, and the work is
 * enqueued on `stream` (a cudaStream_t) without waiting.  Pointers and
 * stream must belong to the current device.  Its scratch memory is one
 * array in the library's static device memory, 24 MiB per device, held
 * until the process exits; volumes of more than 1048576 voxels (1 << 20) are
 * rejected with FIR_ERR_INVALID_ARGUMENT.  The first call on each device
 * looks up the array's address (cudaGetSymbolAddress).  Under CUDA's lazy
 * module loading (the default since CUDA 12.2) that lookup is what reserves
 * the 24 MiB on the device, so a caller that fixes its memory budget at
 * start-up should make one call (or one warm-up call on a small volume) on
 * each device before it reserves its budget, or run with
 * CUDA_MODULE_LOADING=EAGER, which reserves the array when the library is
 * loaded.  Make that first call before any stream capture.
 * All calls on a device share the one array, so calls that can overlap on
 * the GPU (different streams, no ordering between them) race and corrupt
 * each other; order them on one stream.  The accumulator is cleared by each
 * call.  geometry is FIR_GEOMETRY_REFERENCE or FIR_GEOMETRY_EXACT.
 * Device-side checks of non-finite input are not reported by this call. */
fir_status fir_osem_subiteration_noalloc(const fir_proj_desc* proj, const double* crystal_xy,
                                         const double* slice_z, const float* sino, const float* bias,
                                         const fir_vol_desc* vol, float* img, const float* sens_frame,
                                         const fir_osem_params* params, int subset, int subiter,
                                         int geometry, void* stream);

/* The projection/ratio/backprojection half of an OSEM sub-iteration alone
 * (reconAlgos.cc:119-158, also the loop body of OSEM_ResoReco,
 * reconAlgos.cc:273-312): bp is zeroed, then for every bin of subset
 * `subset` of n_subsets, line = projection of img (+ bias), and if line >
 * 1e-5 the ratio sino/line is backprojected into bp.  bias may be NULL. */
fir_status fir_ratio_backprojection(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino,
                                    const float* bias, const fir_vol_desc* vol, const float* img,
                                    float* bp, int n_subsets, int subset);

/* One rank's share of fir_ratio_backprojection when a subset's views are
 * split between n_shards ranks (or GPUs): bp is zeroed, then the views
 * subset + n_subsets * k of the subset with k % n_shards == shard are
 * projected, and the ratio backprojected, exactly as fir_ratio_backprojection
 * does for the whole subset.  The shares of shards 0..n_shards-1 partition
 * the subset for any n_shards (the first shards hold one view more when
 * n_shards does not divide the subset's views), so the sum of their bp is
 * the subset's backprojection up to the order of the float additions.
 * Counterpart: the subset loop of reconAlgos.cc:119-158, split across
 * processes (FIR has one process). */
fir_status fir_ratio_backprojection_shard(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino,
                                          const float* bias, const fir_vol_desc* vol, const float* img, float* bp,
                                          int n_subsets, int subset, int n_shards, int shard);

/* Called by fir_osem after sub-iteration `subiter` when params->save_interval
 * asks for an intermediate image; img is a host copy (nx*ny*nz floats). */
typedef void (*fir_osem_save_fn)(void* user, int subiter, const float* img);

/* reconAlgos::OSEM: the initial cut, then n_iterations x n_subsets
 * sub-iterations.  sens holds n_subsets frames.  save may be NULL. */
fir_status fir_osem(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                    const fir_vol_desc* vol, float* img, const float* sens,
                    const fir_osem_params* params, fir_osem_save_fn save, void* user);

/* Resolution-modelling OSEM: the corrected form of reconAlgos::OSEM_ResoReco
 * (reconAlgos.cc:203-367).  The Gaussian B = operations::convolve(fwhm_xyz,
 * cut_radius) is part of the system model A B:
 * - every sensitivity frame is blurred once, B A_s^T 1;
 * - each sub-iteration projects B x, backprojects measured/estimated, and
 *   blurs the backprojection before the EM update.
 * FIR's version projects x instead of B x (reconAlgos.cc:296) and divides the
 * image rather than the backprojection by the sensitivity (:323).  The
 * post-filter of convolution_interval and the cut are applied as in
 * fir_osem.  With any FWHM <= 0 this is fir_osem. */
fir_status fir_osem_psf(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                        const fir_vol_desc* vol, float* img, const float* sens, const fir_osem_params* params,
                        fir_osem_save_fn save, void* user);

/* reconAlgos::OSEM_ResoReco exactly as FIR runs it (reconAlgos.cc:203-367),
 * with the images kept on the device for the whole run:
 * - the initial cut, then every one of the n_sens_frames (>= n_subsets)
 *   frames of sens is filtered in place, once (FIR's operations::convolve
 *   filters all frames of the sensitivity volume);
 * - per sub-iteration: the ratio backprojection of the unfiltered image
 *   (as fir_ratio_backprojection), the backprojection filtered, then
 *   img <- img / sens[subset] and img <- img * bp with the 1e-5 gates of
 *   VolData's operators, the post-filter every convolution_interval
 *   sub-iterations, and the cut.
 * These are FIR's own steps, including the two that fir_osem_psf corrects
 * (the projection of the unfiltered image, reconAlgos.cc:296, and the
 * division of the image by the sensitivity, :323).  sens is read and
 * written (host buffers are copied back).  save may be NULL. */
fir_status fir_osem_reso_reco(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                              const fir_vol_desc* vol, float* img, float* sens, int n_sens_frames,
                              const fir_osem_params* params, fir_osem_save_fn save, void* user);

/* OSEM with the ordinary-Poisson system model: the mean of bin i is
 * m_i (A x)_i + bias_i, with m the per-bin multiplicative factors
 * (attenuation exp(-A mu) = 1 / ACF, normalisation), instead of FIR's
 * precorrected data with mean (A x)_i + bias_i (reconAlgos.cc:119-158,
 * OSEM.cc:314-338).  Each bin backprojects m_i y_i / (m_i (A x)_i + bias_i)
 * when the denominator exceeds 1e-5.  sino holds the measured counts (not
 * precorrected); sens holds the n_subsets frames A_s^T m (fir_backward of
 * mult).  Float arithmetic: line * m, + bias, y / estimate, * m.  With m = 1
 * this is fir_osem.  No counterpart in FIR, which only precorrects. */
fir_status fir_osem_weighted(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* mult,
                             const float* bias, const fir_vol_desc* vol, float* img, const float* sens,
                             const fir_osem_params* params, fir_osem_save_fn save, void* user);

/* ---- multi-frame projection ----
 *
 * Element type of the multi-frame projectors' data. */
typedef enum fir_dtype
{
  FIR_F32 = 0, /* float data; per frame FIR's arithmetic */
  FIR_F64 = 1  /* double data, double sums and double atomics */
} fir_dtype;

/* Forward projection of the n_frames frames of vol (frame-major images) into
 * n_frames sinograms (frame-major), tracing each LOR once for a group of up to
 * 4 frames.  FIR_F32: frame f's sinogram equals fir_forward of frame f.
 * Counterpart: the frame loop of ForwardProj.cc:79-100 around
 * projections::forward (projections.cc:15-92). */
fir_status fir_forward_frames(fir_ctx* ctx, const fir_vol_desc* vol, const void* img, const fir_proj_desc* proj,
                              void* sino, fir_dtype dtype);
/* Backprojection of n_frames sinograms into the n_frames frames of vol
 * (overwritten): the adjoint of fir_forward_frames.  FIR_F32: frame f equals
 * fir_backward of sinogram f with one subset, up to the order of the float
 * atomic additions.  Counterpart: projections::backward (projections.cc:94-184)
 * once per frame. */
fir_status fir_backward_frames(fir_ctx* ctx, const fir_proj_desc* proj, const void* sino, const fir_vol_desc* vol,
                               void* img, fir_dtype dtype);

/* ---- batched OSEM: many independent reconstructions at once ----
 *
 * No counterpart in FIR, which reconstructs one problem per process.  A
 * batch holds n problems, each with its own scanner, sinogram geometry,
 * volume (one frame) and OSEM parameters, of any sizes.  fir_batch_osem runs
 * reconAlgos::OSEM (reconAlgos.cc:63-201) on all of them together: step t
 * performs sub-iteration t of every problem that has one, with one
 * persistent launch for the projection/backprojection of all those
 * problems' LORs and one launch per image operation for all their images.
 * The schedule can be captured once in a CUDA graph and replayed.  Each
 * problem's result is that of fir_osem on it, up to the order of the float
 * atomic additions of the backprojection.
 *
 * The batch owns device copies of all its data (sinograms, sensitivities,
 * optional biases, images, scratch) and runs on a stream of its own, ordered
 * after and before the context's stream: work queued on the context's
 * stream before fir_batch_osem runs before it, and work queued after it
 * runs after it.  The context's geometry and skip-zero options at creation
 * apply. */
typedef struct fir_batch fir_batch;

fir_status fir_batch_create(fir_batch** batch, fir_ctx* ctx, int n_problems, const fir_scanner_desc* scanners,
                            const fir_proj_desc* projs, const fir_vol_desc* vols, const fir_osem_params* params);
fir_status fir_batch_destroy(fir_batch* batch);
/* Copies problem p's measured sinogram, its sensitivity (n_subsets frames)
 * and its bias sinogram (NULL: none) into the batch; host or device
 * pointers; returns when the copies are done. */
fir_status fir_batch_set_data(fir_batch* batch, int p, const float* sino, const float* sens, const float* bias);
fir_status fir_batch_set_image(fir_batch* batch, int p, const float* img);
/* Waits for the batch's work and reports device-side check failures. */
fir_status fir_batch_get_image(fir_batch* batch, int p, float* img);
/* Launch shape of the projector: threads per block (32..256, a multiple of
 * 32), resident blocks per SM (0: one warp per bundle of 32 LORs, no
 * persistence; otherwise a persistent grid of that many blocks per SM,
 * capped at what fits), and bundles taken per queue access (1..64). */
fir_status fir_batch_set_launch(fir_batch* batch, int block, int blocks_per_sm, int grab);
fir_status fir_batch_get_launch(const fir_batch* batch, int* block, int* blocks_per_sm, int* grab);
/* Shape of the projector's LOR bundles (the 32 LORs one warp traces
 * together): 0 (default), 32 consecutive LORs of the enumeration, i.e.
 * neighbouring tangential bins; A = 1, 2, 4 or 8, tiles of A neighbouring
 * axial planes x 32 / A neighbouring tangential bins of one (segment, view),
 * padded with idle lanes at the planes' edges.  The result is the same for
 * every shape up to the order of the float atomic additions. */
fir_status fir_batch_set_bundle(fir_batch* batch, int axial_tile);
fir_status fir_batch_get_bundle(const fir_batch* batch, int* axial_tile);
/* Autotuner: times the batched projector of the first step that has one
 * (all batched problems' first subsets) for each candidate launch shape
 * (bundle shape, block size, residency, grab) and keeps the fastest; *best_ms
 * (may be NULL) receives its time.  It uses the current images without
 * changing them.  A problem with at least 2^22 LORs per subset, or whose
 * volume fits L2 only as float image and accumulator, is not batched: its
 * projector runs as fir_osem's does, in launches of its own within each step,
 * and the launch shape does not apply to it.  With no batched problem the
 * tuner times nothing, reports no candidates and *best_ms = 0. */
fir_status fir_batch_tune(fir_batch* batch, double* best_ms);
/* The candidates of the last fir_batch_tune with their times: *n receives
 * their number; the first `max` are written to the arrays (each may be
 * NULL): block, blocks_per_sm, grab as fir_batch_set_launch takes them,
 * axial_tile as fir_batch_set_bundle takes it, and the best of two timed
 * runs of step 0's projector in ms. */
fir_status fir_batch_tune_report(const fir_batch* batch, int max, int* block, int* blocks_per_sm, int* grab,
                                 int* axial_tile, double* ms, int* n);
/* Number of steps (the largest number of sub-iterations of any problem) and
 * number of kernel launches of the whole schedule. */
fir_status fir_batch_schedule(const fir_batch* batch, int* n_steps, long long* n_launches);
/* Runs every problem's OSEM (initial cut, then all sub-iterations) in place
 * on the batch's images; asynchronous.  use_graph != 0 captures the schedule
 * in a CUDA graph on first use (and after a launch-shape change) and
 * replays it; 0 launches the kernels one by one. */
fir_status fir_batch_osem(fir_batch* batch, int use_graph);

/* ---- image and sinogram operations ---- */
fir_status fir_em_update(fir_ctx* ctx, const fir_vol_desc* vol, float* img, float* bp,
                         const float* sens_frame);
/* operations::convolve on every frame of vol. */
fir_status fir_convolve(fir_ctx* ctx, const fir_vol_desc* vol, float* img, const float fwhm_xyz[3],
                        float cut_radius);
fir_status fir_cut_circle(fir_ctx* ctx, const fir_vol_desc* vol, float* img, float cut_radius);
fir_status fir_apply_mask(fir_ctx* ctx, const fir_vol_desc* vol, float* img, const float* mask);
fir_status fir_hu_to_mu(fir_ctx* ctx, const fir_vol_desc* vol, float* img);
fir_status fir_proj_exponential(fir_ctx* ctx, const fir_proj_desc* proj, float* sino);
fir_status fir_proj_multiply(fir_ctx* ctx, const fir_proj_desc* proj, float* a, const float* b);

/* ProjData::getBinCoordinates (ProjData.h:96-104, ProjData.cc:342-479) for n
 * LORs.  pairs: n x (ring1, crystal1, ring2, crystal2) ints (a device pointer
 * must be 16-byte aligned).  coords (may be NULL): n x (found, seg, view,
 * axial, tang), found being FIR's return value and the rest zeros where it
 * is 0.  bins (may be NULL): the flat
 * file-order bin index, or -1 where FIR returns false or the coordinates
 * fall outside the sinogram's arrays. */
fir_status fir_bin_coordinates(fir_ctx* ctx, const fir_proj_desc* proj, long long n, const int* pairs, int* coords,
                               long long* bins);
/* ProjData::rebinWeight (ProjData.h:112, ProjData.cc:541-615), in place: for
 * span > 1, every bin of an axial position that merges w > 1 ring
 * differences of one ring sum is multiplied by (float)(1.0 / w); span 1 is a
 * no-op.  FIR indexes these rows through ProjData::getInd, which adds the
 * segment offset twice (ProjData.inl:76-79, ProjHeader.inl:55) and writes
 * outside its arrays once there is more than one segment; here every row the
 * algorithm names is weighted. */
fir_status fir_proj_rebin_weight(fir_ctx* ctx, const fir_proj_desc* proj, float* sino);

/* ---- path dumps (debugging and parity checks) ---- */
/* Siddon::computePath for n segments, ends[6*i..6*i+5] = (x1,y1,z1,x2,y2,z2).
 * Row i of coords/lengths holds up to cap elements; counts[i] = elements of
 * the path (may exceed cap), crosses[i] = 1 if the segment meets the volume. */
fir_status fir_siddon_paths(fir_ctx* ctx, const fir_vol_desc* vol, long long n, const double* ends,
                            int cap, int* coords, double* lengths, int* counts, int* crosses);
/* Same for sinogram bins given by their flat index (file order). */
fir_status fir_lor_paths(fir_ctx* ctx, const fir_proj_desc* proj, const fir_vol_desc* vol,
                         long long n, const long long* bins, int cap, int* coords, double* lengths,
                         int* counts, int* crosses);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* FIR_CUDA_H */
