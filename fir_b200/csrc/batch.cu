// Batched OSEM: the sub-iterations of many independent reconstructions
// (each with its own scanner, sinogram geometry, image and parameters) run
// as one launch per kernel kind.
//
// A launch covers a list of items (problem, subset).  Its work units are
// numbered across the items: bundles of 32 consecutive enumerated LORs of
// one problem for the projector (a bundle never straddles two problems, so
// a warp still traces 32 adjacent, nearly parallel LORs), blocks of
// kBatchBlock voxels of one problem for the image kernels.  A unit finds its
// item by binary search over the items' first units.  All per-problem data
// (geometry, enumeration, tables, buffers, filter taps) is read from the
// BatchProblem array in device memory, so a schedule captured once in a CUDA
// graph stays valid while the data changes.
//
// The projector is persistent: a grid sized to the SMs' resident capacity
// whose warps take bundles from an atomic counter until none are left
// (heavy problems are listed first, so the tail is made of light bundles).
// There is no waiting on other blocks or other warps anywhere: the counter
// is only ever incremented, and a warp that reads a value past the end
// stops.
#include "lor_body.cuh"

namespace fir
{
namespace
{
__device__ __forceinline__ int find_item(const BatchItem* __restrict__ items, int n, int unit)
{
  int lo = 0, hi = n;
  while (hi - lo > 1)
  {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&items[mid].unit_begin) <= unit)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int take(int* queue, int grab, int lane)
{
  int v = 0;
  if (lane == 0)
  {
    v = atomicAdd(queue, grab);
  }
  return __shfl_sync(0xffffffffu, v, 0);
}

// Enumerated index of lane `lane` of bundle j of a tiled launch shape: tile
// (ta, tt) of A axial planes x 32 / A tangential bins in the (segment, view)
// plane of the subset's enumeration; lanes past the plane's edges get
// n_enum (idle).
__device__ __forceinline__ int tiled_lor(const Sino& s, const int* __restrict__ base, int j, int A, int lane)
{
  int lo = 0, hi = s.n_segments;
  while (hi - lo > 1)
  {
    const int mid = (lo + hi) >> 1;
    if (__ldg(base + mid) <= j)
      lo = mid;
    else
      hi = mid;
  }
  const int T = 32 / A;
  const int nax = s.n_axial[lo];
  const int tiles_t = (s.n_tang + T - 1) / T;
  const int per_view = ((nax + A - 1) / A) * tiles_t;
  const int r = j - __ldg(base + lo);
  const int sv = r / per_view;
  const int rem = r - sv * per_view;
  const int ta = rem / tiles_t;
  const int a = ta * A + lane / T;
  const int t = (rem - ta * tiles_t) * T + lane % T;
  if (a >= nax || t >= s.n_tang)
  {
    return s.n_enum;
  }
  return s.enum_base[lo] + (sv * nax + a) * s.n_tang + t;
}

// The projection gathers each problem's double copy.  Problems whose volumes
// fit L2 only as float image and accumulator run fir_osem's kernel in launches
// of their own instead.
template<bool kPersistent>
__global__ void __launch_bounds__(256, 4) k_batch_osem(const BatchProblem* __restrict__ P,
                                                    const BatchItem* __restrict__ items, int n_items,
                                                    int n_bundles, int* queue, int grab, int axial_tile,
                                                    int* check)
{
  const int lane = threadIdx.x & 31;
  int b = kPersistent ? take(queue, grab, lane) : (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  // b is uniform across the warp, so every lane runs the same bundles
  while (b < n_bundles)
  {
    const int end = kPersistent ? min(b + grab, n_bundles) : b + 1;
    for (int k = b; k < end; ++k)
    {
      const int it = find_item(items, n_items, k);
      const int p = __ldg(&items[it].problem);
      const int subset = __ldg(&items[it].subset);
      const BatchProblem& pb = P[p];
      const int j = k - __ldg(&items[it].unit_begin);
      const int i = axial_tile == 0 ? j * 32 + lane : tiled_lor(pb.s, pb.bundle_base, j, axial_tile, lane);
      osem_lor(pb.g, pb.s, subset, pb.t, pb.wide, pb.wide_t, pb.sino, pb.bias, pb.bp, pb.bp_t, pb.skip_zero != 0, i,
               check);
      // lanes whose paths ended early wait here, so that the warp starts the
      // next bundle together instead of splitting across two bundles
      __syncwarp();
    }
    if (!kPersistent)
    {
      break;
    }
    b = take(queue, grab, lane);
  }
}

struct Voxel
{
  const BatchProblem* pb;
  const BatchItem* item;
  int j;  // linear voxel index within the problem; -1 past its end
};

__device__ __forceinline__ Voxel voxel_of(const BatchProblem* P, const BatchItem* items, int n_items)
{
  const int it = find_item(items, n_items, blockIdx.x);
  Voxel v;
  v.item = items + it;
  v.pb = P + __ldg(&items[it].problem);
  v.j = (blockIdx.x - __ldg(&items[it].unit_begin)) * kBatchBlock + threadIdx.x;
  if (v.j >= v.pb->nvox)
  {
    v.j = -1;
  }
  return v;
}

// Index of voxel j in the layout with x and y exchanged.
__device__ __forceinline__ int exchanged(const BatchProblem& pb, int j)
{
  const int x = j % pb.g.nx;
  const int r = j / pb.g.nx;
  const int y = r % pb.g.ny;
  return (r / pb.g.ny * pb.g.nx + x) * pb.g.ny + y;
}

__device__ __forceinline__ double radius_at(const BatchProblem& pb, int j)
{
  const int x = j % pb.g.nx;
  const int y = (j / pb.g.nx) % pb.g.ny;
  return radius_of(x, y, pb.g.nx, pb.g.ny, pb.vx, pb.vy);
}

// operations::cutCircle (operations.cc:187-220) as the start of
// reconAlgos::OSEM (reconAlgos.cc:98-101), and the projector's double copy.
__global__ void __launch_bounds__(kBatchBlock) k_batch_prepare(const BatchProblem* __restrict__ P,
                                                               const BatchItem* __restrict__ items, int n_items,
                                                               int write_img)
{
  const Voxel v = voxel_of(P, items, n_items);
  if (v.j < 0)
  {
    return;
  }
  const BatchProblem& pb = *v.pb;
  float x = pb.img[v.j];
  if (pb.cut > 0.0f && radius_at(pb, v.j) > (double)pb.cut)
  {
    x = 0.0f;
  }
  if (write_img)
  {
    pb.img[v.j] = x;
  }
  if (pb.wide != nullptr)
  {
    pb.wide[v.j] = (double)x;
  }
  pb.bp[v.j] = 0.0f;
  if (pb.bp_t != nullptr)
  {
    const int jt = exchanged(pb, v.j);
    if (pb.wide_t != nullptr)
    {
      pb.wide_t[jt] = (double)x;
    }
    if (pb.img_t != nullptr)
    {
      pb.img_t[jt] = x;
    }
    pb.bp_t[jt] = 0.0f;
  }
}

// reconAlgos.cc:161-166 (VolData::operator/= then operator*=, VolData.cc:
// 305-343), then, for a sub-iteration that does not filter, the cut of
// reconAlgos.cc:180-183.  bp is cleared for the next sub-iteration.
__global__ void __launch_bounds__(kBatchBlock) k_batch_em(const BatchProblem* __restrict__ P,
                                                          const BatchItem* __restrict__ items, int n_items)
{
  const Voxel v = voxel_of(P, items, n_items);
  if (v.j < 0)
  {
    return;
  }
  const BatchProblem& pb = *v.pb;
  const int jt = pb.bp_t != nullptr ? exchanged(pb, v.j) : -1;
  const float b = jt >= 0 ? __fadd_rn(pb.bp[v.j], pb.bp_t[jt]) : pb.bp[v.j];
  const float s = __ldg(pb.sens + (size_t)__ldg(&v.item->subset) * pb.nvox + v.j);
  const float q = ((double)b > kEps && (double)s > kEps) ? __fdiv_rn(b, s) : 0.0f;
  const float x0 = pb.img[v.j];
  float x = ((double)x0 > kEps && (double)q > kEps) ? __fmul_rn(x0, q) : 0.0f;
  pb.bp[v.j] = 0.0f;
  if (jt >= 0)
  {
    pb.bp_t[jt] = 0.0f;
  }
  if (!__ldg(&v.item->filter))
  {
    if (pb.cut > 0.0f && radius_at(pb, v.j) > (double)pb.cut)
    {
      x = 0.0f;
    }
    if (pb.wide != nullptr)
    {
      pb.wide[v.j] = (double)x;
    }
    if (jt >= 0 && pb.wide_t != nullptr)
    {
      pb.wide_t[jt] = (double)x;
    }
    if (jt >= 0 && pb.img_t != nullptr)
    {
      pb.img_t[jt] = x;
    }
  }
  pb.img[v.j] = x;
}

// One pass of operations::convolve (operations.cc:84-156).  The z pass
// finishes the sub-iteration: where r >= cut - 5 fwhm the pre-filter value
// is kept (operations.cc:158-185; the image still holds it, since only this
// thread writes voxel j and the pass reads t2), then the cut.
template<int AXIS>
__global__ void __launch_bounds__(kBatchBlock) k_batch_filter(const BatchProblem* __restrict__ P,
                                                              const BatchItem* __restrict__ items, int n_items)
{
  const Voxel v = voxel_of(P, items, n_items);
  if (v.j < 0)
  {
    return;
  }
  const BatchProblem& pb = *v.pb;
  const int nx = pb.g.nx, ny = pb.g.ny, nz = pb.g.nz;
  const int j = v.j;
  const Taps& taps = AXIS == 0 ? pb.tx : (AXIS == 1 ? pb.ty : pb.tz);
  const float* in = AXIS == 0 ? pb.img : (AXIS == 1 ? pb.t1 : pb.t2);
  const int coord = AXIS == 0 ? j % nx : (AXIS == 1 ? (j / nx) % ny : j / (nx * ny));
  const int len = AXIS == 0 ? nx : (AXIS == 1 ? ny : nz);
  const int stride = AXIS == 0 ? 1 : (AXIS == 1 ? nx : nx * ny);
  const int half = taps.half;
  float sum = 0.0f, norm = 0.0f;
  for (int k = -half; k <= half; ++k)
  {
    const int c = coord + k;
    if (c >= 0 && c < len)
    {
      const float kv = taps.w[half + k];
      sum = __fadd_rn(sum, __fmul_rn(kv, __ldg(in + j + k * stride)));
      norm = __fadd_rn(norm, kv);
    }
  }
  if (AXIS == 0)
  {
    if (norm > 0.0f)
    {
      pb.t1[j] = __fdiv_rn(sum, norm);
    }
  }
  else if (AXIS == 1)
  {
    if (norm > 0.0f)
    {
      pb.t2[j] = __fdiv_rn(sum, norm);
    }
  }
  else
  {
    const float old = pb.img[j];
    float x = norm > 0.0f ? __fdiv_rn(sum, norm) : old;
    if (pb.cut > 0.0f)
    {
      const double r = radius_at(pb, j);
      if (r >= __dsub_rn((double)pb.cut, __dmul_rn(5.0, (double)pb.fwhm)))
      {
        x = old;
      }
      if (r > (double)pb.cut)
      {
        x = 0.0f;
      }
    }
    pb.img[j] = x;
    if (pb.wide != nullptr)
    {
      pb.wide[j] = (double)x;
    }
    if (pb.wide_t != nullptr)
    {
      pb.wide_t[exchanged(pb, j)] = (double)x;
    }
    if (pb.img_t != nullptr)
    {
      pb.img_t[exchanged(pb, j)] = x;
    }
  }
}
}  // namespace

void launch_batch_prepare(const BatchProblem* P, const BatchItem* items, int n_items, int n_units,
                          bool write_img, cudaStream_t stream)
{
  if (n_units > 0)
  {
    k_batch_prepare<<<n_units, kBatchBlock, 0, stream>>>(P, items, n_items, write_img ? 1 : 0);
  }
}

namespace
{
void project(const BatchProblem* P, const BatchItem* items, int n_items, int n_bundles, int* queue,
             const BatchLaunch& L, int n_sms, int* check, cudaStream_t stream)
{
  const long long threads = (long long)n_bundles * 32;
  const long long plain_blocks = (threads + L.block - 1) / L.block;
  if (L.blocks_per_sm <= 0)
  {
    k_batch_osem<false><<<(unsigned)plain_blocks, L.block, 0, stream>>>(P, items, n_items, n_bundles, nullptr, 1,
                                                                         L.axial_tile, check);
    return;
  }
  long long blocks = (long long)n_sms * L.blocks_per_sm;
  if (blocks > plain_blocks)
  {
    blocks = plain_blocks;
  }
  k_batch_osem<true><<<(unsigned)blocks, L.block, 0, stream>>>(P, items, n_items, n_bundles, queue, L.grab,
                                                                L.axial_tile, check);
}
}  // namespace

void launch_batch_project(const BatchProblem* P, const BatchItem* items, int n_items, int n_bundles,
                          int* queue, const BatchLaunch& L, int n_sms, int* check, cudaStream_t stream)
{
  if (n_bundles <= 0)
  {
    return;
  }
  project(P, items, n_items, n_bundles, queue, L, n_sms, check, stream);
}

void launch_batch_em(const BatchProblem* P, const BatchItem* items, int n_items, int n_units, cudaStream_t stream)
{
  if (n_units > 0)
  {
    k_batch_em<<<n_units, kBatchBlock, 0, stream>>>(P, items, n_items);
  }
}

void launch_batch_filter(const BatchProblem* P, const BatchItem* items, int n_items, int n_units, int axis,
                         cudaStream_t stream)
{
  if (n_units <= 0)
  {
    return;
  }
  if (axis == 0)
  {
    k_batch_filter<0><<<n_units, kBatchBlock, 0, stream>>>(P, items, n_items);
  }
  else if (axis == 1)
  {
    k_batch_filter<1><<<n_units, kBatchBlock, 0, stream>>>(P, items, n_items);
  }
  else
  {
    k_batch_filter<2><<<n_units, kBatchBlock, 0, stream>>>(P, items, n_items);
  }
}

long long batch_bundles(const Sino& s, int axial_tile)
{
  if (axial_tile == 0)
  {
    return ((long long)s.n_enum + 31) / 32;
  }
  long long n = 0;
  const int T = 32 / axial_tile;
  const int vps = s.n_views / s.n_subsets;
  for (int k = 0; k < s.n_segments; ++k)
  {
    n += (long long)vps * ((s.n_axial[k] + axial_tile - 1) / axial_tile) * ((s.n_tang + T - 1) / T);
  }
  return n;
}

void batch_bundle_bases(const Sino& s, int axial_tile, int* base)
{
  long long n = 0;
  const int A = axial_tile > 0 ? axial_tile : 1;
  const int T = 32 / A;
  const int vps = s.n_views / s.n_subsets;
  for (int k = 0; k < s.n_segments; ++k)
  {
    base[k] = (int)n;
    n += (long long)vps * ((s.n_axial[k] + A - 1) / A) * ((s.n_tang + T - 1) / T);
  }
  base[s.n_segments] = (int)n;
}

int batch_max_resident(int block)
{
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_osem<true>, block, 0) != cudaSuccess)
  {
    cudaGetLastError();
    return 1;
  }
  return n > 0 ? n : 1;
}
}  // namespace fir
