// Opt-in float traversal of the fused OSEM sub-iteration
// (FIR_OPT_TRAVERSAL = FIR_TRAVERSAL_FLOAT).
//
// FIR traverses every LOR in double precision.  Here FIR's double set-up
// (siddon_setup: entry and exit alphas, first crossings, steps, start voxel)
// is kept and the loop runs in float: alphas and their running sums, the
// minimum, the tie test |alpha - next| < 1e-5 and the lengths, with the
// projection accumulated in float by fused multiply-adds and gathered from
// the float image.  The oracle's precision study measures what this changes
// on the clinical workload: the voxel lists of 2.9 % of the LORs (crossings of
// two dimensions closer than the tie window are merged or split differently)
// and line integrals by up to 1 %.  It is therefore not FIR's traversal and
// never the default; the OSEM images it gives are compared with FIR's in the
// tests.
//
// Work decomposition, warp convergence and the x/y-exchanged images follow
// the exact kernel (projector.cu): one thread per LOR, consecutive threads
// take neighbouring tangential bins, LORs running mostly along x gather from
// and accumulate into images with x and y exchanged.
#include "lor_body.cuh"

namespace fir
{
namespace
{
// State of one float walk.
struct WalkF
{
  float a[3], da[3];
  int step[3], left[3];
  int c, tr;
  float amin, amax, d12;
  float end;  // below this minimum no index can leave the volume
};

// The float state of a walk from FIR's double set-up.  end: every
// dimension's exit crossing a + left * da, computed in double, less EPS and
// a margin of 2^-10 for the rounding of the float running sums.
__device__ __forceinline__ WalkF to_float(const Walk& w)
{
  WalkF f;
  double end = w.amax;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    f.a[d] = (float)w.a[d];
    f.da[d] = (float)w.da[d];
    f.step[d] = w.step[d];
    f.left[d] = w.left[d];
    const double x = w.left[d] > 0 ? dadd(w.a[d], dmul((double)w.left[d], w.da[d])) : w.a[d];
    const double lim = dsub(dsub(x, kEps), dmul(x, 0x1p-10));
    end = (lim < end || lim != lim) ? lim : end;
  }
  f.c = w.c;
  f.tr = w.tr;
  f.amin = (float)w.amin;
  f.amax = (float)w.amax;
  f.d12 = (float)w.d12;
  f.end = (float)end;
  return f;
}

// Advances left in each dimension, from the linear index.
__device__ __forceinline__ void left_from_index(const Grid& g, WalkF& w)
{
  const int z = w.c / g.nxy;
  const int rest = w.c - z * g.nxy;
  const int slow = rest / (w.tr ? g.ny : g.nx);
  const int fast = rest - slow * (w.tr ? g.ny : g.nx);
  const int idx[3] = {w.tr ? slow : fast, w.tr ? fast : slow, z};
  const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    w.left[d] = w.step[d] > 0 ? n[d] - 1 - idx[d] : idx[d];
  }
}

// One step of the computePath loop (Siddon.cc:207-252) in float: emits the
// current voxel (its index is inside the volume) and advances each dimension
// whose crossing lies within 1e-5 of the next alpha.  Returns next alpha.
template<bool kCount, class Emit>
__device__ __forceinline__ float step_float(WalkF& w, float prev, Emit&& emit)
{
  const float m = fminf(w.a[0], fminf(w.a[1], w.a[2]));
  const float next = fminf(m, w.amax);
  emit(w.c, __fmul_rn(__fsub_rn(next, prev), w.d12));
  const float thr = __fadd_rn(next, 1e-5f);
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    if (w.a[d] < thr)
    {
      w.a[d] = __fadd_rn(w.a[d], w.da[d]);
      w.c += w.step[d];
      if (kCount)
      {
        w.left[d] -= 1;
      }
    }
  }
  return next;
}

// The loop, stopping at alphaMax, when an index leaves the volume, or at
// the step bound (only non-finite input reaches it; the return value is
// then false).  As in the exact traversal, the steps below w.end run first
// without the advance counts, which are then rebuilt from the voxel index for
// the checked steps that end the walk.
template<class Emit>
__device__ __forceinline__ bool walk_float(const Grid& g, WalkF w, bool go, Emit&& emit)
{
  float prev = w.amin;
  const bool active = go && prev < w.amax;
  int guard = g.guard;
  if (active)
  {
    while (fminf(w.a[0], fminf(w.a[1], w.a[2])) < w.end && guard > 0)
    {
      prev = step_float<false>(w, prev, emit);
      if (!(fminf(w.a[0], fminf(w.a[1], w.a[2])) < w.end))
      {
        break;
      }
      prev = step_float<false>(w, prev, emit);
      guard -= 2;
    }
    left_from_index(g, w);
  }
  bool more = active;
  while (more)
  {
    const float m = fminf(w.a[0], fminf(w.a[1], w.a[2]));
    prev = step_float<true>(w, prev, emit);
    --guard;
    more = m < w.amax && (w.left[0] | w.left[1] | w.left[2]) >= 0 && guard > 0;
  }
  return !go || guard > 0;
}

// One OSEM sub-iteration over the subset of s (reconAlgos.cc:119-158) with
// the float loop: line = projection of img (+ bias); if line > 1e-5 the
// ratio sino / line is backprojected along the same path.
__global__ void __launch_bounds__(256, 4) k_osem_subset_float(Grid g, Sino s, Tables t,
                                                            const float* __restrict__ img,
                                                            const float* __restrict__ img_t,
                                                            const float* __restrict__ sino,
                                                            const float* __restrict__ bias, float* bp, float* bp_t,
                                                            int skip_zero, int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = false;
  const int ie = enum_index(s, i, valid);
  Lor l{};
  Walk w{};
  bool go = false;
  bool tr = false;
  float y = 0.0f;
  if (valid)
  {
    l = decode_bin(s, ie);
    y = __ldg(sino + l.bin);
    if (!(skip_zero && y == 0.0f))
    {
      double e[6];
      lor_ends(s, t, l, e);
      tr = img_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
      go = siddon_setup(g, e, w, tr);
    }
  }
  const WalkF wf = to_float(w);
  const float* im = tr ? img_t : img;
  float* b = tr ? bp_t : bp;
  __builtin_assume(__isGlobal(b));
  float line = 0.0f;
  // each gather is issued two steps before its value is accumulated, so its
  // latency overlaps the walk of those steps; the sum is the same, term by
  // term in order
  float l0 = 0.0f, v0 = 0.0f, l1 = 0.0f, v1 = 0.0f;
  bool ok = walk_float(g, wf, go, [&](int c, float len) {
    line = __fmaf_rn(l0, v0, line);
    l0 = l1;
    v0 = v1;
    l1 = len;
    v1 = __ldg(im + c);
  });
  line = __fmaf_rn(l0, v0, line);
  line = __fmaf_rn(l1, v1, line);
  __syncwarp();
  if (valid && bias != nullptr)
  {
    line = __fadd_rn(line, __ldg(bias + l.bin));
  }
  const bool back = go && ok && (double)line > kEps;
  const float q = back ? __fdiv_rn(y, line) : 0.0f;
  ok = walk_float(g, wf, back, [&](int c, float len) { atomicAdd(b + c, __fmul_rn(len, q)); }) && ok;
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
}

// The float image with x and y exchanged ([z][x][y]), through 32 x 32 tiles
// in shared memory.
constexpr int kXTile = 32, kXRows = 8;

__global__ void __launch_bounds__(kXTile * kXRows) k_exchange_float(int nx, int ny, int nz,
                                                                   const float* __restrict__ in,
                                                                   float* __restrict__ out_t)
{
  __shared__ float tile[kXTile][kXTile + 1];
  const int x0 = blockIdx.x * kXTile, y0 = blockIdx.y * kXTile;
  for (int z = blockIdx.z; z < nz; z += gridDim.z)
  {
    const size_t plane = (size_t)nx * ny * z;
    for (int j = threadIdx.y; j < kXTile; j += kXRows)
    {
      const int x = x0 + threadIdx.x, y = y0 + j;
      if (x < nx && y < ny)
      {
        tile[j][threadIdx.x] = in[plane + (size_t)y * nx + x];
      }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kXTile; j += kXRows)
    {
      const int y = y0 + threadIdx.x, x = x0 + j;
      if (x < nx && y < ny)
      {
        out_t[plane + (size_t)x * ny + y] = tile[threadIdx.x][j];
      }
    }
    __syncthreads();
  }
}
}  // namespace

void launch_exchange_float(int nx, int ny, int nz, const float* in, float* out_t, const LaunchCfg& cfg)
{
  if ((long long)nx * ny * nz <= 0)
  {
    return;
  }
  const dim3 grid((unsigned)((nx + kXTile - 1) / kXTile), (unsigned)((ny + kXTile - 1) / kXTile),
                  (unsigned)(nz < 64 ? nz : 64));
  k_exchange_float<<<grid, dim3(kXTile, kXRows), 0, cfg.stream>>>(nx, ny, nz, in, out_t);
}

void launch_osem_subset_float(const Grid& g, const Sino& s, const Tables& t, const float* img, const float* img_t,
                              const float* sino, const float* bias, float* bp, float* bp_t, bool skip_zero,
                              const LaunchCfg& cfg)
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
  const unsigned nb = (unsigned)((s.n_enum + cfg.block - 1) / cfg.block);
  k_osem_subset_float<<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, img, img_t, sino, bias, bp, bp_t,
                                                        skip_zero ? 1 : 0, cfg.check);
}
}  // namespace fir
