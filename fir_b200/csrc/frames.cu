// Multi-frame projection: several images projected (or sinograms
// backprojected) with one traversal per LOR.
//
// FIR projects a multi-frame volume frame by frame (ForwardProj.cc:79-100),
// tracing every path once per frame.  Here a thread traces its LOR once and
// gathers (or scatters) all frames of a group of up to 4 at every step.  The
// frames of a group are interleaved in device scratch, voxel-major
// ([voxel][frame], stride FMAX), so the frames of one voxel share one or two
// 32-byte sectors: the traversal, which dominates the cost, is paid once per
// group instead of once per frame.
//
// Two arithmetics:
// * FIR_F32: per frame exactly fir_forward / fir_backward (float running sum
//   widened and rounded per step; float atomics of float(len * value));
// * FIR_F64: double data, double running sums and double atomics, for
//   gradient checks that need more than float resolution.
#include "lor_body.cuh"

namespace fir
{
namespace
{
// Vector float reductions in global memory (sm_90 and later); the address
// is 16-byte (v4) or 8-byte (v2) aligned and converted to the global space.
__device__ __forceinline__ void red_add_v4(float* p, float a, float b, float c, float d)
{
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(__cvta_generic_to_global(p)), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

__device__ __forceinline__ void red_add_v2(float* p, float a, float b)
{
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(__cvta_generic_to_global(p)), "f"(a), "f"(b) : "memory");
}

// Four doubles from a 32-byte aligned global address in one 256-bit load
// (sm_100): the L1 serves a lane's whole sector in one wavefront, where two
// 128-bit loads took two.
__device__ __forceinline__ void ld_v4(const double* p, double* x)
{
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(x[0]), "=d"(x[1]), "=d"(x[2]), "=d"(x[3])
      : "l"(__cvta_generic_to_global(p)));
}

template<int FMAX, bool F64>
__global__ void __launch_bounds__(256, 4) k_forward_frames(Grid g, Sino s, Tables t, const double* __restrict__ il,
                                                        const double* __restrict__ il_t, int nf, long long n_bins,
                                                        void* out, int* check)
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
    tr = il_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
    go = siddon_setup(g, e, w, tr);
  }
  const double* src = tr ? il_t : il;
  float lf[FMAX];
  double ld[FMAX];
#pragma unroll
  for (int f = 0; f < FMAX; ++f)
  {
    lf[f] = 0.0f;
    ld[f] = 0.0;
  }
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      double x[FMAX];
      if (FMAX == 1)
      {
        x[0] = __ldg(src + c);
      }
      else if (FMAX == 4)
      {
        // a voxel's 4 frames are one 32-byte sector: one 256-bit load
        ld_v4(src + (size_t)c * 4, x);
      }
      else
      {
        // a voxel's frames are 16-byte aligned: FMAX doubles at c * FMAX
        const double2* v = reinterpret_cast<const double2*>(src + (size_t)c * FMAX);
#pragma unroll
        for (int k = 0; k < FMAX / 2; ++k)
        {
          const double2 q = __ldg(v + k);
          x[2 * k] = q.x;
          x[2 * k + 1] = q.y;
        }
      }
#pragma unroll
      for (int f = 0; f < FMAX; ++f)
      {
        if (f < nf)
        {
          if (F64)
            ld[f] = dadd(ld[f], dmul(len, x[f]));
          else
            lf[f] = accumulate(lf[f], len, x[f]);
        }
      }
    }
  });
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
  if (valid)
  {
#pragma unroll
    for (int f = 0; f < FMAX; ++f)
    {
      if (f < nf)
      {
        if (F64)
          static_cast<double*>(out)[f * n_bins + l.bin] = ld[f];
        else
          static_cast<float*>(out)[f * n_bins + l.bin] = lf[f];
      }
    }
  }
}

template<int FMAX, bool F64>
__global__ void __launch_bounds__(256, 4) k_backward_frames(Grid g, Sino s, Tables t, const void* __restrict__ sino,
                                                         int nf, long long n_bins, void* acc_n, void* acc_t,
                                                         int skip_zero, int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  Walk w{};
  bool go = false;
  bool tr = false;
  double v[FMAX];
#pragma unroll
  for (int f = 0; f < FMAX; ++f)
  {
    v[f] = 0.0;
  }
  if (i < s.n_enum)
  {
    const Lor l = decode_bin(s, i);
    bool any = false;
#pragma unroll
    for (int f = 0; f < FMAX; ++f)
    {
      if (f < nf)
      {
        v[f] = F64 ? __ldg(static_cast<const double*>(sino) + f * n_bins + l.bin)
                   : (double)__ldg(static_cast<const float*>(sino) + f * n_bins + l.bin);
        any = any || v[f] != 0.0;
      }
    }
    // with every value 0 every contribution is exactly 0
    if (!(skip_zero && !any))
    {
      double e[6];
      lor_ends(s, t, l, e);
      tr = acc_t != nullptr && fabs(dsub(e[3], e[0])) > fabs(dsub(e[4], e[1]));
      go = siddon_setup(g, e, w, tr);
    }
  }
  void* acc = tr ? acc_t : acc_n;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      if (F64 || FMAX == 1)
      {
#pragma unroll
        for (int f = 0; f < FMAX; ++f)
        {
          if (f < nf)
          {
            if (F64)
              atomicAdd(static_cast<double*>(acc) + (size_t)c * FMAX + f, dmul(len, v[f]));
            else
              atomicAdd(static_cast<float*>(acc) + (size_t)c * FMAX + f, __double2float_rn(dmul(len, v[f])));
          }
        }
      }
      else
      {
        // vector reductions: one L2 atomic for the 2 or 4 frames.  Each element
        // still receives float(len * value); padding frames (f >= nf, value
        // 0) receive 0 in slots nothing reads.
        float q[FMAX];
#pragma unroll
        for (int f = 0; f < FMAX; ++f)
        {
          q[f] = __double2float_rn(dmul(len, v[f]));
        }
        float* a = static_cast<float*>(acc) + (size_t)c * FMAX;
        if (FMAX == 2)
        {
          red_add_v2(a, q[0], q[1]);
        }
        else
        {
#pragma unroll
          for (int k = 0; k < FMAX / 4; ++k)
          {
            red_add_v4(a + 4 * k, q[4 * k], q[4 * k + 1], q[4 * k + 2], q[4 * k + 3]);
          }
        }
      }
    }
  });
  if (!ok)
  {
    flag(check, kCheckWalkGuard);
  }
}

// Index of voxel j in the layout with x and y exchanged ([z][x][y]).
__device__ __forceinline__ long long exchanged(long long j, int nx, int ny)
{
  const long long r = j / nx;
  const int x = (int)(j - r * nx);
  const long long z = r / ny;
  const int y = (int)(r - z * ny);
  return (z * nx + x) * ny + y;
}

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// il[j * fmax + f] = frame f of img at voxel j (widened), 0 for f >= nf;
// il_t (when given) the same with x and y exchanged.
template<typename T>
__global__ void k_interleave(long long nvox, int nf, int fmax, int nx, int ny, const T* __restrict__ img,
                             double* __restrict__ il, double* __restrict__ il_t)
{
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nvox * fmax)
  {
    return;
  }
  const long long j = k / fmax;
  const int f = (int)(k - j * fmax);
  const double v = f < nf ? (double)img[(size_t)f * nvox + j] : 0.0;
  il[k] = v;
  if (il_t != nullptr)
  {
    il_t[exchanged(j, nx, ny) * fmax + f] = v;
  }
}

// img[f][j] = acc[j * fmax + f] (+ the exchanged accumulator's value) for
// f < nf.
template<typename T>
__global__ void k_deinterleave(long long nvox, int nf, int fmax, int nx, int ny, const T* __restrict__ acc,
                               const T* __restrict__ acc_t, T* __restrict__ img)
{
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nvox * nf)
  {
    return;
  }
  const int f = (int)(k / nvox);
  const long long j = k - (long long)f * nvox;
  const T a = acc[j * fmax + f];
  img[k] = acc_t != nullptr ? add_rn(a, acc_t[exchanged(j, nx, ny) * fmax + f]) : a;
}

unsigned blocks_for(long long n, int block)
{
  return (unsigned)((n + block - 1) / block);
}

template<int FMAX>
void fwd(const Grid& g, const Sino& s, const Tables& t, const double* il, const double* il_t, int nf,
         long long n_bins, void* out, bool f64, const LaunchCfg& cfg)
{
  const unsigned nb = blocks_for(s.n_enum, cfg.block);
  if (f64)
    k_forward_frames<FMAX, true><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, il, il_t, nf, n_bins, out, cfg.check);
  else
    k_forward_frames<FMAX, false><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, il, il_t, nf, n_bins, out, cfg.check);
}

template<int FMAX>
void bwd(const Grid& g, const Sino& s, const Tables& t, const void* sino, int nf, long long n_bins, void* acc,
         void* acc_t, bool f64, bool skip_zero, const LaunchCfg& cfg)
{
  const unsigned nb = blocks_for(s.n_enum, cfg.block);
  if (f64)
    k_backward_frames<FMAX, true><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, sino, nf, n_bins, acc, acc_t,
                                                                     skip_zero ? 1 : 0, cfg.check);
  else
    k_backward_frames<FMAX, false><<<nb, cfg.block, 0, cfg.stream>>>(g, s, t, sino, nf, n_bins, acc, acc_t,
                                                                      skip_zero ? 1 : 0, cfg.check);
}
}  // namespace

int frames_stride(int nf)
{
  return nf <= 1 ? 1 : (nf <= 2 ? 2 : kMaxFramesPerPass);
}

void launch_interleave(long long nvox, int nf, int nx, int ny, const void* img, bool f64, double* il, double* il_t,
                       const LaunchCfg& cfg)
{
  const int fmax = frames_stride(nf);
  const unsigned nb = blocks_for(nvox * fmax, 256);
  if (f64)
    k_interleave<double><<<nb, 256, 0, cfg.stream>>>(nvox, nf, fmax, nx, ny, static_cast<const double*>(img), il,
                                                     il_t);
  else
    k_interleave<float><<<nb, 256, 0, cfg.stream>>>(nvox, nf, fmax, nx, ny, static_cast<const float*>(img), il, il_t);
}

void launch_deinterleave(long long nvox, int nf, int nx, int ny, const void* acc, const void* acc_t, bool f64,
                         void* img, const LaunchCfg& cfg)
{
  const int fmax = frames_stride(nf);
  const unsigned nb = blocks_for(nvox * nf, 256);
  if (f64)
    k_deinterleave<double><<<nb, 256, 0, cfg.stream>>>(nvox, nf, fmax, nx, ny, static_cast<const double*>(acc),
                                                       static_cast<const double*>(acc_t), static_cast<double*>(img));
  else
    k_deinterleave<float><<<nb, 256, 0, cfg.stream>>>(nvox, nf, fmax, nx, ny, static_cast<const float*>(acc),
                                                      static_cast<const float*>(acc_t), static_cast<float*>(img));
}

void launch_forward_frames(const Grid& g, const Sino& s, const Tables& t, const double* il, const double* il_t, int nf,
                           long long n_bins, void* out, bool f64, const LaunchCfg& cfg)
{
  if (s.n_enum == 0 || nf <= 0)
  {
    return;
  }
  switch (frames_stride(nf))
  {
    case 1: fwd<1>(g, s, t, il, il_t, nf, n_bins, out, f64, cfg); break;
    case 2: fwd<2>(g, s, t, il, il_t, nf, n_bins, out, f64, cfg); break;
    default: fwd<kMaxFramesPerPass>(g, s, t, il, il_t, nf, n_bins, out, f64, cfg); break;
  }
}

void launch_backward_frames(const Grid& g, const Sino& s, const Tables& t, const void* sino, int nf,
                            long long n_bins, void* acc, void* acc_t, bool f64, bool skip_zero, const LaunchCfg& cfg)
{
  if (s.n_enum == 0 || nf <= 0)
  {
    return;
  }
  switch (frames_stride(nf))
  {
    case 1: bwd<1>(g, s, t, sino, nf, n_bins, acc, acc_t, f64, skip_zero, cfg); break;
    case 2: bwd<2>(g, s, t, sino, nf, n_bins, acc, acc_t, f64, skip_zero, cfg); break;
    default: bwd<kMaxFramesPerPass>(g, s, t, sino, nf, n_bins, acc, acc_t, f64, skip_zero, cfg); break;
  }
}
}  // namespace fir
