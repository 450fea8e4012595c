// Internal interface between the C ABI (capi.cu) and the kernels
// (projector.cu, image_ops.cu).  Not installed; not part of the ABI.
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "siddon.cuh"

namespace fir
{
// Bits of the per-context device check word.
enum DeviceCheck : int
{
  kCheckWalkGuard = 1,  // a traversal hit its iteration bound (non-finite input)
};

enum class FwdEpilogue
{
  None,
  Exp  // ProjData::exponential applied to the line integral (ACF)
};

struct LaunchCfg
{
  int block;
  cudaStream_t stream;
  int* check;  // device check word
};

// projector.cu
// img_t (or null): the image with x and y exchanged ([z][x][y]), which LORs
// running mostly along x use; the caller adds a backprojected img_t into img.
void launch_forward(const Grid& g, const Sino& s, const Tables& t, const double* img, const double* img_t,
                    float* sino, FwdEpilogue ep, const LaunchCfg& cfg);
void launch_backward(const Grid& g, const Sino& s, const Tables& t, const float* sino, float* img, float* img_t,
                     bool skip_zero, const LaunchCfg& cfg);
// mult: per-bin multiplicative factors of the ordinary-Poisson model, or
// nullptr for FIR's model.
// img_t / bp_t: the image and the accumulator with x and y exchanged (both
// or neither); LORs running mostly along x use them.
void launch_osem_subset(const Grid& g, const Sino& s, const Tables& t, const double* img, const double* img_t,
                        const float* sino, const float* mult, const float* bias, float* bp, float* bp_t,
                        bool skip_zero, const LaunchCfg& cfg);
// The same, gathering from the float image itself; with the exchanged float
// image and accumulator (img_t, bp_t, both or neither) as two launches, one
// per orientation.
void launch_osem_subset_float_image(const Grid& g, const Sino& s, const Tables& t, const float* img,
                                    const float* img_t, const float* sino, const float* mult, const float* bias,
                                    float* bp, float* bp_t, bool skip_zero, const LaunchCfg& cfg);
// compact.cu: the enumerated indices of s (list null) whose bin of sino is
// not 0, ascending, into list (s.n_enum entries), their number into *count
// (device memory).  With temp null only *temp_bytes is set (CUB convention).
cudaError_t launch_nonzero_list(const Sino& s, const float* sino, int* list, int* count, void* temp,
                                size_t* temp_bytes, const LaunchCfg& cfg);
// fast.cu: the opt-in float traversal of the fused OSEM kernel.
void launch_osem_subset_float(const Grid& g, const Sino& s, const Tables& t, const float* img, const float* img_t,
                              const float* sino, const float* bias, float* bp, float* bp_t, bool skip_zero,
                              const LaunchCfg& cfg);
void launch_exchange_float(int nx, int ny, int nz, const float* in, float* out_t, const LaunchCfg& cfg);
void launch_siddon_paths(const Grid& g, long long n, const double* ends, int cap, int* coords,
                         double* lengths, int* counts, int* crosses, const LaunchCfg& cfg);
void launch_lor_paths(const Grid& g, const Sino& s, const Tables& t, long long n,
                      const long long* bins, int cap, int* coords, double* lengths, int* counts,
                      int* crosses, const LaunchCfg& cfg);

// deterministic.cu
// ratio[i] = sino / (projection + bias) for enumerated LOR i, or 0
// (with mult: m * sino / (m * projection + bias)); counts (or null): the
// pair counts deterministic_backproject needs for that ratio.
void launch_ratio(const Grid& g, const Sino& s, const Tables& t, const double* img, const float* sino,
                  const float* mult, const float* bias, float* ratio, int* counts, const LaunchCfg& cfg);
// Device scratch of at least `bytes` for slot 0 (per-LOR counts and
// offsets) or slot 1 (pairs and sort space); nullptr if unavailable.
using ScratchFn = std::function<void*(int slot, size_t bytes)>;
// img += backprojection of vals (per bin, or per enumerated LOR; nullptr =
// all ones), summed in FIR's serial LOR order with FIR's rounding, in
// chunks of at most max_pairs_cap (voxel, product) pairs.  counts_in (or
// null): per-LOR pair counts from launch_ratio for these vals.  Synchronises
// the stream once, after counting.
cudaError_t deterministic_backproject(const Grid& g, const Sino& s, const Tables& t, const float* vals,
                                      bool vals_by_enum, const int* counts_in, float* img, const ScratchFn& scratch,
                                      long long max_pairs_cap, long long n_vox, const LaunchCfg& cfg,
                                      long long* launches);

// image_ops.cu
constexpr int kMaxHalfTaps = 64;
struct Taps
{
  int half;
  float w[2 * kMaxHalfTaps + 1];
};
void launch_em_update(long long n, float* img, float* bp, const float* sens, const LaunchCfg& cfg);
// The same after adding the x/y-exchanged accumulator bp_t into bp (one
// launch in place of launch_merge_oriented and launch_em_update).
void launch_em_update_oriented(int nx, int ny, int nz, float* img, float* bp, const float* bp_t, const float* sens,
                               const LaunchCfg& cfg);
void launch_em_update_image_first(long long n, float* img, const float* bp, const float* sens,
                                  const LaunchCfg& cfg);
// Exact widening of a float image to double for the projector gathers.
void launch_widen(long long n, const float* in, double* out, const LaunchCfg& cfg);
// Double copies of an [nz][ny][nx] image: out in the same layout, out_t as
// [nz][nx][ny].
void launch_widen_oriented(int nx, int ny, int nz, const float* in, double* out, double* out_t,
                           const LaunchCfg& cfg);
// bp[z][y][x] += bp_t[z][x][y].
void launch_merge_oriented(int nx, int ny, int nz, float* bp, const float* bp_t, const LaunchCfg& cfg);
// One separable pass of operations::convolve along axis (0=x, 1=y, 2=z).
void launch_conv_pass(int nx, int ny, int nz, int axis, const Taps& taps, const float* in, float* out,
                      const LaunchCfg& cfg);
// Restore voxels with r >= cut - 5*fwhm from the pre-filter copy.
void launch_conv_restore(int nx, int ny, int nz, double vx, double vy, float limit_base, float fwhm,
                         const float* copy, float* img, const LaunchCfg& cfg);
void launch_cut_circle(int nx, int ny, int nz, double vx, double vy, float cut_radius, float* img,
                       const LaunchCfg& cfg);
void launch_apply_mask(long long n, float* img, const float* mask, const LaunchCfg& cfg);
void launch_hu_to_mu(long long n, float* img, const LaunchCfg& cfg);
void launch_exponential(long long n, float* sino, const LaunchCfg& cfg);
void launch_proj_multiply(long long n, float* a, const float* b, const LaunchCfg& cfg);
// ProjData::getBinCoordinates on n (ring1, crystal1, ring2, crystal2) int4
// pairs (16-byte aligned); coords (5 ints per pair: flag, seg, view, axial,
// tang) and bins may be nullptr.
void launch_bin_coordinates(const Sino& s, int max_ring_diff, long long n, const int* pairs, int* coords,
                            long long* bins, const LaunchCfg& cfg);
// sino *= table[segment][axial] where the factor is not 1 (s: one subset).
void launch_rebin_weight(const Sino& s, const float* table, int max_axial, float* sino, const LaunchCfg& cfg);

// Distance of voxel (x, y)'s centre from the volume axis, in FIR's double
// arithmetic (operations.cc:160-185 and :206-212).
__device__ __forceinline__ double radius_of(int x, int y, int nx, int ny, double vx, double vy)
{
  const double px = __dsub_rn(__dadd_rn(__dmul_rn((double)x, vx), __ddiv_rn(vx, 2.0)),
                              __ddiv_rn(__dmul_rn((double)nx, vx), 2.0));
  const double py = __dsub_rn(__dadd_rn(__dmul_rn((double)y, vy), __ddiv_rn(vy, 2.0)),
                              __ddiv_rn(__dmul_rn((double)ny, vy), 2.0));
  return __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
}

// batch.cu: many independent OSEM problems per launch.
// One problem of a batch, resident in device memory.
struct BatchProblem
{
  Grid g;
  Sino s;  // enumeration for the problem's number of subsets (subset unused)
  Tables t;
  const float* sino;
  const float* bias;  // nullptr: none
  const float* sens;  // n_subsets frames
  float* img;
  double* wide;  // double copy of img for the projector gathers (null: it gathers img itself)
  float* bp;
  // wide, img and bp with x and y exchanged ([z][x][y]), for LORs running
  // mostly along x; bp_t is added into bp by the EM step.  Problems with the
  // double copy have wide_t, those that gather floats img_t (null: none).
  double* wide_t;
  float* bp_t;
  float* img_t;
  float* t1;
  float* t2;
  int nvox;
  int skip_zero;
  double vx, vy;
  float cut;   // cut radius (0: none)
  float fwhm;  // max(fwhm x, fwhm y), for the filter's edge restore
  Taps tx, ty, tz;
  // bundles of the launch shape's tiled form (axial_tile > 0): first bundle
  // of each segment of one subset's enumeration
  int bundle_base[kMaxSegments + 1];
};

// One problem's share of one batched launch.  Work units are numbered
// across the items of a launch: bundles of 32 LORs for the projector,
// blocks of kBatchBlock voxels for the image kernels.
struct BatchItem
{
  int problem;
  int subset;
  int filter;  // 1: the sub-iteration filters the image (the filter passes finish it)
  int unit_begin;
};

constexpr int kBatchBlock = 256;

struct BatchLaunch
{
  int block;          // threads per block of the projector
  int blocks_per_sm;  // 0: a warp per bundle, no persistence
  int grab;           // bundles taken per queue access by a persistent warp
  // shape of a bundle (the 32 LORs of a warp): 0, 32 consecutive enumerated
  // LORs; A = 1, 2, 4 or 8, a tile of A axial planes x 32 / A tangential
  // bins of one (segment, view), padded at the plane's edges
  int axial_tile;
};

// Bundles of one subset of a problem with the given axial tile (0: linear).
long long batch_bundles(const Sino& s, int axial_tile);
void batch_bundle_bases(const Sino& s, int axial_tile, int* base);

// wide = cut(img), bp = 0 (and img = cut(img) when write_img).
void launch_batch_prepare(const BatchProblem* P, const BatchItem* items, int n_items, int n_units,
                          bool write_img, cudaStream_t stream);
// bp += backprojection of measured/estimated for every item's subset.
// queue: a zeroed counter (persistent mode).  The items' problems gather
// their double copies (wide).
void launch_batch_project(const BatchProblem* P, const BatchItem* items, int n_items, int n_bundles,
                          int* queue, const BatchLaunch& L, int n_sms, int* check, cudaStream_t stream);
// Gated EM update of img; bp <- 0.  Items without filtering also apply the
// cut and refresh wide.
void launch_batch_em(const BatchProblem* P, const BatchItem* items, int n_items, int n_units,
                     cudaStream_t stream);
// Filter pass along axis (0: img -> t1, 1: t1 -> t2, 2: t2 -> img with the
// edge restore, the cut and the refresh of wide).
void launch_batch_filter(const BatchProblem* P, const BatchItem* items, int n_items, int n_units, int axis,
                         cudaStream_t stream);
// Resident blocks per SM of the projector at this block size.
int batch_max_resident(int block);

// frames.cu: several frames per traversal, in groups of up to kMaxFramesPerPass
// (measured on B200 at 8 frames of a clinical sinogram: two groups of 4 run
// faster than one of 8, whose kernels need more registers).
constexpr int kMaxFramesPerPass = 4;
// Interleave stride of a group of nf frames: 1, 2, 4 or 8.
int frames_stride(int nf);
// il[j * stride + f] = (double) frame f of img (float or double, frame-major);
// il_t (or null) the same with x and y exchanged.
void launch_interleave(long long nvox, int nf, int nx, int ny, const void* img, bool f64, double* il, double* il_t,
                       const LaunchCfg& cfg);
// img[f][j] = acc[j * stride + f] (+ acc_t at the exchanged index when
// given; float or double).
void launch_deinterleave(long long nvox, int nf, int nx, int ny, const void* acc, const void* acc_t, bool f64,
                         void* img, const LaunchCfg& cfg);
// out[f * n_bins + bin] = projection of frame f (float or double sinograms).
// LORs running mostly along x gather from il_t when it is given.
void launch_forward_frames(const Grid& g, const Sino& s, const Tables& t, const double* il, const double* il_t, int nf,
                           long long n_bins, void* out, bool f64, const LaunchCfg& cfg);
// acc[c * stride + f] += backprojection of sino[f * n_bins + ...]; LORs
// running mostly along x add into acc_t (x and y exchanged) when it is given.
void launch_backward_frames(const Grid& g, const Sino& s, const Tables& t, const void* sino, int nf,
                            long long n_bins, void* acc, void* acc_t, bool f64, bool skip_zero, const LaunchCfg& cfg);
}  // namespace fir
