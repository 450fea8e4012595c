// Image-space and sinogram-space element-wise kernels of the OSEM loop:
// the gated EM update, the separable Gaussian filter with edge
// renormalisation, the cylindrical cut, the mask, HU to mu conversion, and the
// sinogram exponential / product.  All float arithmetic uses explicit
// round-to-nearest intrinsics (no FMA contraction) in FIR's operation order,
// so results are bit-identical to FIR's.
#include "internal.h"

namespace fir
{
namespace
{
constexpr int kBlock = 256;

unsigned blocks_for(long long n, int block = kBlock)
{
  return (unsigned)((n + block - 1) / block);
}

// VolData::operator/= then VolData::operator*= (VolData.cc:305-343), as used
// by reconAlgos.cc:161-166: bp <- bp/sens and img <- img*bp, each gated by
// both operands exceeding 1e-5.  bp is left holding the quotient.
__global__ void k_em_update(long long n, float* __restrict__ img, float* __restrict__ bp,
                            const float* __restrict__ sens)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n)
  {
    return;
  }
  const float b = bp[i];
  const float s = __ldg(sens + i);
  const float q = ((double)b > kEps && (double)s > kEps) ? __fdiv_rn(b, s) : 0.0f;
  const float x = img[i];
  img[i] = ((double)x > kEps && (double)q > kEps) ? __fmul_rn(x, q) : 0.0f;
  bp[i] = q;
}

// The EM step of OSEM_ResoReco as FIR runs it (reconAlgos.cc:320-326):
// img <- img/sens, then img <- img*bp, each with VolData's 1e-5 gates
// (VolData.cc:305-343); the image, not the backprojection, is divided.
__global__ void k_em_update_image_first(long long n, float* __restrict__ img, const float* __restrict__ bp,
                                        const float* __restrict__ sens)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n)
  {
    return;
  }
  const float s = __ldg(sens + i);
  const float b = __ldg(bp + i);
  float x = img[i];
  x = ((double)x > kEps && (double)s > kEps) ? __fdiv_rn(x, s) : 0.0f;
  x = ((double)x > kEps && (double)b > kEps) ? __fmul_rn(x, b) : 0.0f;
  img[i] = x;
}

__global__ void k_widen(long long n, const float* __restrict__ in, double* __restrict__ out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n)
  {
    out[i] = (double)in[i];
  }
}

// The two orientations of the projector's images move through 32 x 32
// tiles of one plane in shared memory, so that both layouts are read and
// written in whole rows.
constexpr int kTile = 32;
constexpr int kTileRows = 8;

// out[z][y][x] = in[z][y][x] and out_t[z][x][y] = in[z][y][x], widened to
// double (exact).
__global__ void __launch_bounds__(kTile * kTileRows) k_widen_oriented(int nx, int ny, int nz,
                                                                      const float* __restrict__ in,
                                                                      double* __restrict__ out,
                                                                      double* __restrict__ out_t)
{
  __shared__ float tile[kTile][kTile + 1];
  const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
  for (int z = blockIdx.z; z < nz; z += gridDim.z)
  {
    const size_t plane = (size_t)nx * ny * z;
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int x = x0 + threadIdx.x, y = y0 + j;
      if (x < nx && y < ny)
      {
        const size_t k = plane + (size_t)y * nx + x;
        const float v = in[k];
        out[k] = (double)v;
        tile[j][threadIdx.x] = v;
      }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int y = y0 + threadIdx.x, x = x0 + j;
      if (x < nx && y < ny)
      {
        out_t[plane + (size_t)x * ny + y] = (double)tile[threadIdx.x][j];
      }
    }
    __syncthreads();
  }
}

// bp[z][y][x] += bp_t[z][x][y] (one float addition per voxel).
__global__ void __launch_bounds__(kTile * kTileRows) k_merge_oriented(int nx, int ny, int nz, float* __restrict__ bp,
                                                                      const float* __restrict__ bp_t)
{
  __shared__ float tile[kTile][kTile + 1];
  const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
  for (int z = blockIdx.z; z < nz; z += gridDim.z)
  {
    const size_t plane = (size_t)nx * ny * z;
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int x = x0 + j, y = y0 + threadIdx.x;
      if (x < nx && y < ny)
      {
        tile[j][threadIdx.x] = bp_t[plane + (size_t)x * ny + y];
      }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int y = y0 + j, x = x0 + threadIdx.x;
      if (x < nx && y < ny)
      {
        const size_t k = plane + (size_t)y * nx + x;
        bp[k] = __fadd_rn(bp[k], tile[threadIdx.x][j]);
      }
    }
    __syncthreads();
  }
}

// k_em_update with the exchanged accumulator added first: b = bp[z][y][x] +
// bp_t[z][x][y] (the float addition of k_merge_oriented), then the gated
// division and product of k_em_update; bp is left holding the quotient.
__global__ void __launch_bounds__(kTile * kTileRows) k_em_update_oriented(int nx, int ny, int nz,
                                                                          float* __restrict__ img,
                                                                          float* __restrict__ bp,
                                                                          const float* __restrict__ bp_t,
                                                                          const float* __restrict__ sens)
{
  __shared__ float tile[kTile][kTile + 1];
  const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
  for (int z = blockIdx.z; z < nz; z += gridDim.z)
  {
    const size_t plane = (size_t)nx * ny * z;
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int x = x0 + j, y = y0 + threadIdx.x;
      if (x < nx && y < ny)
      {
        tile[j][threadIdx.x] = bp_t[plane + (size_t)x * ny + y];
      }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kTile; j += kTileRows)
    {
      const int y = y0 + j, x = x0 + threadIdx.x;
      if (x < nx && y < ny)
      {
        const size_t k = plane + (size_t)y * nx + x;
        const float b = __fadd_rn(bp[k], tile[threadIdx.x][j]);
        const float sv = __ldg(sens + k);
        const float q = ((double)b > kEps && (double)sv > kEps) ? __fdiv_rn(b, sv) : 0.0f;
        const float v = img[k];
        img[k] = ((double)v > kEps && (double)q > kEps) ? __fmul_rn(v, q) : 0.0f;
        bp[k] = q;
      }
    }
    __syncthreads();
  }
}

dim3 plane_tiles(int nx, int ny, int nz)
{
  return dim3((unsigned)((nx + kTile - 1) / kTile), (unsigned)((ny + kTile - 1) / kTile),
              (unsigned)(nz < 65535 ? nz : 65535));
}

// One pass of operations::convolve (operations.cc:84-156) along AXIS: sum
// and weight norm over the in-bounds taps, accumulated in float in tap order,
// then sum / norm.  Threads cover the xy plane (blockIdx.x) of slices
// blockIdx.y, blockIdx.y + gridDim.y, ...; volumes hold fewer than 2^31
// voxels (checked on the host), so 32-bit indices suffice and x, y come from
// one division.
template<int AXIS>
__global__ void __launch_bounds__(256) k_conv_pass(int nx, int ny, int nz, Taps taps, const float* __restrict__ in,
                                                   float* __restrict__ out)
{
  const int nxy = nx * ny;
  const int ixy = blockIdx.x * blockDim.x + threadIdx.x;
  if (ixy >= nxy)
  {
    return;
  }
  const int y = ixy / nx;
  const int x = ixy - y * nx;
  const int len = AXIS == 0 ? nx : (AXIS == 1 ? ny : nz);
  const int stride = AXIS == 0 ? 1 : (AXIS == 1 ? nx : nxy);
  for (int z = blockIdx.y; z < nz; z += gridDim.y)
  {
    const int i = z * nxy + ixy;
    const int coord = AXIS == 0 ? x : (AXIS == 1 ? y : z);
    float sum = 0.0f, norm = 0.0f;
    for (int k = -taps.half; k <= taps.half; ++k)
    {
      const int c = coord + k;
      if (c >= 0 && c < len)
      {
        const float kv = taps.w[taps.half + k];
        sum = __fadd_rn(sum, __fmul_rn(kv, __ldg(in + i + k * stride)));
        norm = __fadd_rn(norm, kv);
      }
    }
    if (norm > 0.0f)
    {
      out[i] = __fdiv_rn(sum, norm);
    }
  }
}

__global__ void k_conv_restore(int nx, int ny, int nz, double vx, double vy, float cut, float fwhm,
                               const float* __restrict__ copy, float* __restrict__ img)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx * ny * nz)
  {
    return;
  }
  const int x = i % nx;
  const int y = (i / nx) % ny;
  // cutRadius - 5.0 * fwhm: float cut radius widened, double product.
  if (radius_of(x, y, nx, ny, vx, vy) >= __dsub_rn((double)cut, __dmul_rn(5.0, (double)fwhm)))
  {
    img[i] = copy[i];
  }
}

__global__ void k_cut_circle(int nx, int ny, int nz, double vx, double vy, float cut, float* img)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx * ny * nz)
  {
    return;
  }
  const int x = i % nx;
  const int y = (i / nx) % ny;
  if (radius_of(x, y, nx, ny, vx, vy) > (double)cut)
  {
    img[i] = 0.0f;
  }
}

// operations::applyMask (operations.cc:222-241).
__global__ void k_apply_mask(long long n, float* img, const float* __restrict__ mask)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n && __ldg(mask + i) <= 0.0f)
  {
    img[i] = 0.0f;
  }
}

// operations::HounsfieldToMuMap (operations.cc:243-284): piecewise linear,
// float arithmetic, water mu = 0.0096/mm.
__global__ void k_hu_to_mu(long long n, float* img)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n)
  {
    return;
  }
  const float water = 0.0096f;
  const float s1 = __fdiv_rn(water, 1000.0f);
  const float s2 = __fdiv_rn(__fsub_rn(0.015f, water), 1000.0f);
  float v = img[i];
  if ((double)v <= -1000.0)
  {
    v = 0.0f;
  }
  else if ((double)v <= 0.0)
  {
    v = __fadd_rn(__fmul_rn(v, s1), water);
  }
  else
  {
    v = __fadd_rn(__fmul_rn(v, s2), water);
  }
  img[i] = v;
}

// ProjData::exponential (ProjData.cc:514-539).
__global__ void k_exponential(long long n, float* sino)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n)
  {
    const float v = sino[i];
    sino[i] = (double)v > kEps ? __double2float_rn(exp((double)v)) : 1.0f;
  }
}

// ProjData::operator*= (ProjData.cc:481-512).
__global__ void k_proj_multiply(long long n, float* a, const float* __restrict__ b)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n)
  {
    const float x = a[i], y = __ldg(b + i);
    a[i] = ((double)x > kEps && (double)y > kEps) ? __fmul_rn(x, y) : 0.0f;
  }
}
// ProjData::getBinCoordinates on n crystal pairs; coords[5i..] = FIR's
// result flag, seg, view, axial, tang (zeros where the flag is 0), bins[i] =
// flat file-order
// index, or -1 where FIR returns false or the coordinates fall outside the
// sinogram's arrays.
__global__ void k_bin_coordinates(Sino s, int max_ring_diff, long long n, const int4* __restrict__ pairs,
                                  int* coords, long long* bins)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n)
  {
    return;
  }
  const int4 q = pairs[i];
  int c[4] = {0, 0, 0, 0};
  const bool ok = bin_of_crystals(s, max_ring_diff, q.x, q.y, q.z, q.w, c);
  long long flat = -1;
  if (ok)
  {
    const int si = c[0] + s.seg_offset;
    if (si >= 0 && si < s.n_segments && c[1] >= 0 && c[1] < s.n_views && c[2] >= 0 && c[2] < s.n_axial[si])
    {
      flat = (long long)s.seg_base[si] + ((long long)c[1] * s.n_axial[si] + c[2]) * s.n_tang + c[3] + s.tang_offset;
    }
  }
  if (coords != nullptr)
  {
    coords[5 * i] = ok ? 1 : 0;
    coords[5 * i + 1] = ok ? c[0] : 0;
    coords[5 * i + 2] = ok ? c[1] : 0;
    coords[5 * i + 3] = ok ? c[2] : 0;
    coords[5 * i + 4] = ok ? c[3] : 0;
  }
  if (bins != nullptr)
  {
    bins[i] = flat;
  }
}

// ProjData::rebinWeight: bin *= factor of its (segment, axial) row, for the
// rows whose factor is not 1 (table: n_segments x max_axial floats).
__global__ void k_rebin_weight(Sino s, const float* __restrict__ table, int max_axial, float* sino)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_enum)
  {
    return;
  }
  const Lor l = decode_bin(s, i);
  const float f = __ldg(table + (l.seg + s.seg_offset) * max_axial + l.axial);
  if (f != 1.0f)
  {
    sino[l.bin] = __fmul_rn(sino[l.bin], f);
  }
}
}  // namespace

void launch_em_update(long long n, float* img, float* bp, const float* sens, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_em_update<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, img, bp, sens);
  }
}

void launch_em_update_image_first(long long n, float* img, const float* bp, const float* sens,
                                  const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_em_update_image_first<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, img, bp, sens);
  }
}

void launch_widen(long long n, const float* in, double* out, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_widen<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, in, out);
  }
}

void launch_widen_oriented(int nx, int ny, int nz, const float* in, double* out, double* out_t,
                           const LaunchCfg& cfg)
{
  if ((long long)nx * ny * nz > 0)
  {
    k_widen_oriented<<<plane_tiles(nx, ny, nz), dim3(kTile, kTileRows), 0, cfg.stream>>>(nx, ny, nz, in, out, out_t);
  }
}

void launch_merge_oriented(int nx, int ny, int nz, float* bp, const float* bp_t, const LaunchCfg& cfg)
{
  if ((long long)nx * ny * nz > 0)
  {
    k_merge_oriented<<<plane_tiles(nx, ny, nz), dim3(kTile, kTileRows), 0, cfg.stream>>>(nx, ny, nz, bp, bp_t);
  }
}

void launch_em_update_oriented(int nx, int ny, int nz, float* img, float* bp, const float* bp_t, const float* sens,
                               const LaunchCfg& cfg)
{
  if ((long long)nx * ny * nz > 0)
  {
    k_em_update_oriented<<<plane_tiles(nx, ny, nz), dim3(kTile, kTileRows), 0, cfg.stream>>>(nx, ny, nz, img, bp,
                                                                                             bp_t, sens);
  }
}

void launch_conv_pass(int nx, int ny, int nz, int axis, const Taps& taps, const float* in, float* out,
                      const LaunchCfg& cfg)
{
  const long long n = (long long)nx * ny * nz;
  if (n <= 0)
  {
    return;
  }
  const dim3 grid(blocks_for((long long)nx * ny), (unsigned)(nz < 65535 ? nz : 65535));
  if (axis == 0)
  {
    k_conv_pass<0><<<grid, kBlock, 0, cfg.stream>>>(nx, ny, nz, taps, in, out);
  }
  else if (axis == 1)
  {
    k_conv_pass<1><<<grid, kBlock, 0, cfg.stream>>>(nx, ny, nz, taps, in, out);
  }
  else
  {
    k_conv_pass<2><<<grid, kBlock, 0, cfg.stream>>>(nx, ny, nz, taps, in, out);
  }
}

void launch_conv_restore(int nx, int ny, int nz, double vx, double vy, float cut, float fwhm,
                         const float* copy, float* img, const LaunchCfg& cfg)
{
  const long long n = (long long)nx * ny * nz;
  if (n > 0)
  {
    k_conv_restore<<<blocks_for(n), kBlock, 0, cfg.stream>>>(nx, ny, nz, vx, vy, cut, fwhm, copy, img);
  }
}

void launch_cut_circle(int nx, int ny, int nz, double vx, double vy, float cut, float* img,
                       const LaunchCfg& cfg)
{
  const long long n = (long long)nx * ny * nz;
  if (n > 0)
  {
    k_cut_circle<<<blocks_for(n), kBlock, 0, cfg.stream>>>(nx, ny, nz, vx, vy, cut, img);
  }
}

void launch_apply_mask(long long n, float* img, const float* mask, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_apply_mask<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, img, mask);
  }
}

void launch_hu_to_mu(long long n, float* img, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_hu_to_mu<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, img);
  }
}

void launch_exponential(long long n, float* sino, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_exponential<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, sino);
  }
}

void launch_proj_multiply(long long n, float* a, const float* b, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_proj_multiply<<<blocks_for(n), kBlock, 0, cfg.stream>>>(n, a, b);
  }
}

void launch_bin_coordinates(const Sino& s, int max_ring_diff, long long n, const int* pairs, int* coords,
                            long long* bins, const LaunchCfg& cfg)
{
  if (n > 0)
  {
    k_bin_coordinates<<<blocks_for(n), kBlock, 0, cfg.stream>>>(s, max_ring_diff, n,
                                                                reinterpret_cast<const int4*>(pairs), coords, bins);
  }
}

void launch_rebin_weight(const Sino& s, const float* table, int max_axial, float* sino, const LaunchCfg& cfg)
{
  if (s.n_enum > 0)
  {
    k_rebin_weight<<<blocks_for(s.n_enum), kBlock, 0, cfg.stream>>>(s, table, max_axial, sino);
  }
}
}  // namespace fir
