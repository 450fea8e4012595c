// Per-LOR device bodies shared by the single-problem kernels (projector.cu)
// and the batched persistent kernel (batch.cu).
#pragma once

#include "internal.h"

namespace fir
{
__device__ __forceinline__ void flag(int* check, int bit)
{
  if (check != nullptr)
  {
    atomicOr(check, bit);
  }
}

// The per-LOR body of one OSEM sub-iteration (reconAlgos.cc:119-158 with
// getLine :11-59) for enumerated index i of `subset`: project the current
// image along the LOR, add the bias, and if the estimate exceeds 1e-5
// backproject measured/estimated along the same path.  The path is
// traversed twice from the same saved setup, so both traversals visit
// identical voxels with identical lengths.  Every lane of the warp must call
// this (lanes with i >= n_enum are idle), since it re-converges the warp
// between the traversals.
//
// kWeighted: the ordinary-Poisson model with multiplicative factors m
// (attenuation, normalisation) per bin: estimate m * line + bias, and the
// backprojected value m * measured / estimate.  Without it the body is FIR's.
//
// img_t and bp_t (both given, or both null) are the same images with x and
// y exchanged.  A LOR that runs mostly along x gathers from img_t and adds
// into bp_t: the 32 parallel LORs of a warp are then offset along the
// contiguous axis, so each warp-wide gather and atomic touches about half as
// many cache lines.  The caller adds bp_t back into bp.  orient 0 (1) limits
// the call to the LORs of the first (second, exchanged) orientation, so that
// two launches each keep one orientation's images in L2; -1 takes both.
//
// TImg: the image the projection gathers from, the double copy or the float
// image itself (widened per step, exact; for volumes whose double copy does
// not fit in L2 beside the accumulator).
template<bool kWeighted, typename TImg = double>
__device__ __forceinline__ void osem_lor_body(const Grid& g, const Sino& s, int subset, const Tables& t,
                                              const TImg* __restrict__ img, const TImg* __restrict__ img_t,
                                              const float* __restrict__ sino, const float* __restrict__ mult,
                                              const float* __restrict__ bias, float* bp, float* bp_t,
                                              bool skip_zero, int i, int* check, int orient = -1)
{
  bool valid = false;
  const int ie = enum_index(s, i, valid);
  Lor l{};
  Walk w{};
  bool go = false;
  bool tr = false;
  float y = 0.0f;
  if (valid)
  {
    l = decode_bin(s, ie, subset);
    y = __ldg(sino + l.bin);
    // With y == 0 the ratio is exactly 0 whatever the estimate, so the bin
    // contributes nothing: skipping it is exact.
    if (!(skip_zero && y == 0.0f))
    {
      double e[6];
      lor_ends(s, t, l, e);
      tr = img_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
      // orient 0 or 1: this launch takes only the LORs of that orientation
      if (orient < 0 || (tr ? 1 : 0) == orient)
      {
        go = siddon_setup(g, e, w, tr);
      }
    }
  }
  const TImg* im = tr ? img_t : img;
  float* b = tr ? bp_t : bp;
  // b may come from a descriptor in memory, not a kernel parameter: without
  // this the compiler cannot tell the atomic's address space and tests it at
  // every step.
  __builtin_assume(__isGlobal(b));
  // Each gather is issued one step before its term is accumulated, so its
  // latency overlaps a step of the walk.  The terms are added in the same
  // order; the first call adds 0 * 0 to the zero sum, which leaves it 0.
  float line = 0.0f;
  double pl = 0.0, pv = 0.0;
  bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      line = accumulate(line, pl, pv);
      pl = len;
      pv = (double)__ldg(im + c);
    }
  });
  line = accumulate(line, pl, pv);
  __syncwarp();
  const float m = kWeighted && valid ? __ldg(mult + l.bin) : 1.0f;
  if (kWeighted)
  {
    line = __fmul_rn(line, m);
  }
  if (valid && bias != nullptr)
  {
    line = __fadd_rn(line, __ldg(bias + l.bin));
  }
  const bool back = go && ok && (double)line > kEps;
  float q = back ? __fdiv_rn(y, line) : 0.0f;
  if (kWeighted)
  {
    q = __fmul_rn(q, m);
  }
  const double ratio = (double)q;
  ok = siddon_walk(g, w, back, [&](bool inside, int c, double len) {
         if (inside)
         {
           atomicAdd(b + c, __double2float_rn(dmul(len, ratio)));
         }
       }) && ok;
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
}
// FIR's sub-iteration body (reconAlgos.cc:119-158).
__device__ __forceinline__ void osem_lor(const Grid& g, const Sino& s, int subset, const Tables& t,
                                         const double* __restrict__ img, const double* __restrict__ img_t,
                                         const float* __restrict__ sino, const float* __restrict__ bias, float* bp,
                                         float* bp_t, bool skip_zero, int i, int* check)
{
  osem_lor_body<false>(g, s, subset, t, img, img_t, sino, nullptr, bias, bp, bp_t, skip_zero, i, check);
}
}  // namespace fir
