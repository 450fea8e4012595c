// Ray-driven projector kernels: forward projection (gather), backprojection
// and sensitivity (scatter), the fused OSEM sub-iteration, and path dumps.
//
// Work decomposition: one thread per line of response.  Consecutive threads
// take consecutive bins of FIR's enumeration, i.e. neighbouring tangential
// bins of one view and axial plane, so a warp holds a bundle of 32 nearly
// parallel, adjacent LORs: their traversals have near-equal trip counts and
// touch neighbouring voxels, which keeps the gathers and scatters of a warp
// step within a few L1/L2 sectors.  Kernels never return early: every lane
// reaches every traversal (lanes without work pass go = false), so warps
// stay converged and __syncwarp() between two traversals is safe.  Paths are
// recomputed on the fly (no LOR cache, no stored path).  The image is
// gathered from a double-precision copy (exact widening of the float image,
// made once per call), which stays resident in the 126 MB L2.  While both fit
// in L2, LORs running mostly along x gather from (and backproject into) a
// copy with x and y exchanged: a warp's parallel LORs are then offset along
// the contiguous axis in either case, and its accesses touch about half as
// many cache lines.
#include "lor_body.cuh"

namespace fir
{
namespace
{
// projections::forward (projections.cc:15-92) with
// VolData::computeLineIntegral (VolData.cc:357-371); optional epilogue
// ProjData::exponential (ProjData.cc:514-539).
// LORs running mostly along x gather from img_t (x and y exchanged) when
// it is given.
template<FwdEpilogue EP>
__global__ void __launch_bounds__(256, 4) k_forward(Grid g, Sino s, Tables t,
                                                 const double* __restrict__ img,
                                                 const double* __restrict__ img_t,
                                                 float* __restrict__ sino, int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < s.n_enum;
  Lor l{};
  Walk w{};
  bool go = false;
  bool tr = false;
  if (valid)
  {
    l = decode_bin(s, i);
    double e[6];
    lor_ends(s, t, l, e);
    tr = img_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
    go = siddon_setup(g, e, w, tr);
  }
  const double* im = tr ? img_t : img;
  float line = 0.0f;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      line = accumulate(line, len, __ldg(im + c));
    }
  });
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
  if (valid)
  {
    if (EP == FwdEpilogue::Exp)
    {
      // exp evaluated in double and rounded once: the correctly rounded float
      // exponential that FIR's std::exp(float) returns (ProjData.cc:531).
      line = (double)line > kEps ? __double2float_rn(exp((double)line)) : 1.0f;
    }
    sino[l.bin] = line;
  }
}

// projections::backward (projections.cc:94-184) with
// VolData::projectLineIntegral (VolData.cc:373-385).  sino == nullptr is the
// all-ones sinogram of computeSensitivityVol (projections.cc:186-197).
// LORs running mostly along x add into img_t (x and y exchanged) when it is
// given.
__global__ void __launch_bounds__(256) k_backward(Grid g, Sino s, Tables t,
                                                  const float* __restrict__ sino, float* img, float* img_t,
                                                  int skip_zero, int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  Walk w{};
  bool go = false;
  bool tr = false;
  double v = 0.0;
  bool valid = false;
  const int ie = enum_index(s, i, valid);
  if (valid)
  {
    const Lor l = decode_bin(s, ie);
    const float val = sino != nullptr ? __ldg(sino + l.bin) : 1.0f;
    v = (double)val;
    // with val == 0 every contribution is exactly 0
    if (!(skip_zero && val == 0.0f))
    {
      double e[6];
      lor_ends(s, t, l, e);
      tr = img_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
      go = siddon_setup(g, e, w, tr);
    }
  }
  float* acc = tr ? img_t : img;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      atomicAdd(acc + c, __double2float_rn(dmul(len, v)));
    }
  });
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
}

// One OSEM sub-iteration over the subset of s: one thread per enumerated
// LOR (reconAlgos.cc:119-158); kWeighted adds the multiplicative factors.
template<bool kWeighted, typename TImg>
__global__ void __launch_bounds__(256, 4) k_osem_subset(Grid g, Sino s, Tables t,
                                                        const TImg* __restrict__ img,
                                                        const TImg* __restrict__ img_t,
                                                        const float* __restrict__ sino,
                                                        const float* __restrict__ mult,
                                                        const float* __restrict__ bias, float* bp, float* bp_t,
                                                        int skip_zero, int* check, int orient)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  osem_lor_body<kWeighted, TImg>(g, s, s.subset, t, img, img_t, sino, mult, bias, bp, bp_t, skip_zero != 0, i,
                                 check, orient);
}

// Path dump of one segment into row i of coords / lengths.
__device__ __forceinline__ void dump_path(const Grid& g, const Walk& w, bool go, long long i, int cap,
                                          int* coords, double* lengths, int* counts, int* crosses,
                                          bool valid, int* check)
{
  int k = 0;
  int* co = coords + i * cap;
  double* le = lengths + i * cap;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      if (k < cap)
      {
        co[k] = c;
        le[k] = len;
      }
      ++k;
    }
  });
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
  if (valid)
  {
    counts[i] = k;
    crosses[i] = go ? 1 : 0;
  }
}

__global__ void k_siddon_paths(Grid g, long long n, const double* __restrict__ ends, int cap,
                               int* coords, double* lengths, int* counts, int* crosses, int* check)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool valid = i < n;
  Walk w{};
  bool go = false;
  if (valid)
  {
    double e[6];
#pragma unroll
    for (int k = 0; k < 6; ++k)
    {
      e[k] = ends[6 * i + k];
    }
    go = siddon_setup(g, e, w);
  }
  dump_path(g, w, go, i, cap, coords, lengths, counts, crosses, valid, check);
}

__global__ void k_lor_paths(Grid g, Sino s, Tables t, long long n, const long long* __restrict__ bins,
                            int cap, int* coords, double* lengths, int* counts, int* crosses,
                            int* check)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool valid = i < n;
  Walk w{};
  bool go = false;
  if (valid)
  {
    // bins are flat file-order indices: enumerated with one subset
    const long long b = bins[i];
    if (b >= 0 && b < s.n_enum)
    {
      const Lor l = decode_bin(s, (int)b);
      double e[6];
      lor_ends(s, t, l, e);
      go = siddon_setup(g, e, w);
    }
  }
  dump_path(g, w, go, i, cap, coords, lengths, counts, crosses, valid, check);
}

unsigned blocks_for(long long n, int block)
{
  return (unsigned)((n + block - 1) / block);
}
}  // namespace

void launch_forward(const Grid& g, const Sino& s, const Tables& t, const double* img, const double* img_t,
                    float* sino, FwdEpilogue ep, const LaunchCfg& cfg)
{
  if (s.n_enum == 0)
  {
    return;
  }
  const unsigned nb = blocks_for(s.n_enum, cfg.block);
  if (ep == FwdEpilogue::Exp)
  {
    k_forward<FwdEpilogue::Exp><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, cfg.check);
  }
  else
  {
    k_forward<FwdEpilogue::None><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, cfg.check);
  }
}

void launch_backward(const Grid& g, const Sino& s, const Tables& t, const float* sino, float* img, float* img_t,
                     bool skip_zero, const LaunchCfg& cfg)
{
  if (s.n_enum == 0)
  {
    return;
  }
  k_backward<<<blocks_for(s.n_enum, cfg.block), cfg.block, 0, cfg.stream>>>(
    g, s, t, sino, img, img_t, skip_zero ? 1 : 0, cfg.check);
}

void launch_osem_subset(const Grid& g, const Sino& s, const Tables& t, const double* img, const double* img_t,
                        const float* sino, const float* mult, const float* bias, float* bp, float* bp_t,
                        bool skip_zero, const LaunchCfg& cfg)
{
  if (s.n_enum == 0)
  {
    return;
  }
  if (img_t == nullptr || bp_t == nullptr)
  {
    img_t = nullptr;
    bp_t = nullptr;
  }
  const unsigned nb = blocks_for(s.n_enum, cfg.block);
  if (mult != nullptr)
  {
    k_osem_subset<true, double><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, mult, bias, bp, bp_t,
                                                                  skip_zero ? 1 : 0, cfg.check, -1);
  }
  else
  {
    k_osem_subset<false, double><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, nullptr, bias, bp,
                                                                   bp_t, skip_zero ? 1 : 0, cfg.check, -1);
  }
}

void launch_osem_subset_float_image(const Grid& g, const Sino& s, const Tables& t, const float* img,
                                    const float* img_t, const float* sino, const float* mult, const float* bias,
                                    float* bp, float* bp_t, bool skip_zero, const LaunchCfg& cfg)
{
  if (s.n_enum == 0)
  {
    return;
  }
  if (img_t == nullptr || bp_t == nullptr)
  {
    img_t = nullptr;
    bp_t = nullptr;
  }
  const unsigned nb = blocks_for(s.n_enum, cfg.block);
  // with the exchanged images: one launch per orientation
  const int first = img_t != nullptr ? 0 : -1, last = img_t != nullptr ? 1 : -1;
  for (int o = first; o <= last; ++o)
  {
    if (mult != nullptr)
    {
      k_osem_subset<true, float><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, mult, bias, bp, bp_t,
                                                                   skip_zero ? 1 : 0, cfg.check, o);
    }
    else
    {
      k_osem_subset<false, float><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, nullptr, bias, bp,
                                                                    bp_t, skip_zero ? 1 : 0, cfg.check, o);
    }
  }
}

void launch_siddon_paths(const Grid& g, long long n, const double* ends, int cap, int* coords,
                         double* lengths, int* counts, int* crosses, const LaunchCfg& cfg)
{
  if (n == 0)
  {
    return;
  }
  k_siddon_paths<<<blocks_for(n, 128), 128, 0, cfg.stream>>>(g, n, ends, cap, coords, lengths, counts,
                                                             crosses, cfg.check);
}

void launch_lor_paths(const Grid& g, const Sino& s, const Tables& t, long long n,
                      const long long* bins, int cap, int* coords, double* lengths, int* counts,
                      int* crosses, const LaunchCfg& cfg)
{
  if (n == 0)
  {
    return;
  }
  k_lor_paths<<<blocks_for(n, 128), 128, 0, cfg.stream>>>(g, s, t, n, bins, cap, coords, lengths, counts,
                                                          crosses, cfg.check);
}
}  // namespace fir
