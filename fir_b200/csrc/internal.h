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
void launch_forward(const Grid& g, const Sino& s, const Tables& t, const double* img, float* sino,
                    FwdEpilogue ep, const LaunchCfg& cfg);
void launch_backward(const Grid& g, const Sino& s, const Tables& t, const float* sino, float* img,
                     bool skip_zero, const LaunchCfg& cfg);
void launch_osem_subset(const Grid& g, const Sino& s, const Tables& t, const double* img,
                        const float* sino, const float* bias, float* bp, bool skip_zero,
                        const LaunchCfg& cfg);
void launch_siddon_paths(const Grid& g, long long n, const double* ends, int cap, int* coords,
                         double* lengths, int* counts, int* crosses, const LaunchCfg& cfg);
void launch_lor_paths(const Grid& g, const Sino& s, const Tables& t, long long n,
                      const long long* bins, int cap, int* coords, double* lengths, int* counts,
                      int* crosses, const LaunchCfg& cfg);

// deterministic.cu
// ratio[i] = sino / (projection + bias) for enumerated LOR i, or 0
void launch_ratio(const Grid& g, const Sino& s, const Tables& t, const double* img, const float* sino,
                  const float* bias, float* ratio, const LaunchCfg& cfg);
// Device scratch of at least `bytes` for slot 0 (per-LOR counts and
// offsets) or slot 1 (pairs and sort space); nullptr if unavailable.
using ScratchFn = std::function<void*(int slot, size_t bytes)>;
// img += backprojection of vals (per bin, or per enumerated LOR; nullptr =
// all ones), summed in FIR's serial LOR order with FIR's rounding, in
// chunks of at most max_pairs_cap (voxel, product) pairs.  Synchronises the
// stream once, after counting.
cudaError_t deterministic_backproject(const Grid& g, const Sino& s, const Tables& t, const float* vals,
                                      bool vals_by_enum, float* img, const ScratchFn& scratch,
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
// Exact widening of a float image to double for the projector gathers.
void launch_widen(long long n, const float* in, double* out, const LaunchCfg& cfg);
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
}  // namespace fir
