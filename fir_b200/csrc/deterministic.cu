// Deterministic backprojection: FIR's serial summation order, reproduced.
//
// FIR adds every contribution to its voxel as voxel = float(double(voxel) +
// length * value) (VolData.cc:373-385).  With float atomics the result
// depends on the order in which LORs reach a voxel.  Here every contribution
// becomes a (voxel, product) pair, written at an offset that follows FIR's
// serial loop order: LORs in enumeration order (subset, segment, view of the
// subset, axial plane, tangential bin; LORCache.cc:10-81), then path order.
// A path visits a voxel at most once.  A stable radix sort on the voxel
// index alone (32-bit keys, only the bits the volume needs) therefore leaves
// each voxel's run in FIR's LOR order, and one thread per run accumulates it
// with FIR's rounding.  The result equals a single-threaded FIR run bit for
// bit, and is independent of scheduling.
//
// Work is chunked over contiguous ranges of LORs; chunks are reduced in
// order, each run continuing from the voxel's value after the previous
// chunk, so chunking does not change the order either.
//
// Each LOR's pairs fill a multiple of 8 slots: the last group is padded with
// pairs whose key is one past the last voxel.  The stable sort puts them in
// one final run, which the reduction skips.  With padded regions a lane
// stages 8 pairs in shared memory and writes them as whole sectors; the
// lanes of a warp start together and emit one pair per step, so their groups
// mostly fill on the same steps.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "internal.h"

namespace fir
{
namespace
{
// Number of elements FIR would store for each enumerated LOR (0 for LORs
// whose value is exactly 0: their products are 0 and leave every voxel
// unchanged, +0 + -0 included, since accumulators start at +0).
__global__ void __launch_bounds__(256) k_count(Grid g, Sino s, Tables t, const float* __restrict__ vals,
                                               int vals_by_enum, int* counts, int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < s.n_enum;
  Walk w{};
  bool go = false;
  if (valid)
  {
    const Lor l = decode_bin(s, i);
    const float v = vals == nullptr ? 1.0f : __ldg(vals + (vals_by_enum ? i : l.bin));
    if (v != 0.0f)
    {
      double e[6];
      lor_ends(s, t, l, e);
      go = siddon_setup(g, e, w);
    }
  }
  int k = 0;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int, double) { k += inside ? 1 : 0; });
  if (!ok && check != nullptr)
  {
    atomicOr(check, kCheckWalkGuard);
  }
  if (valid)
  {
    counts[i] = (k + 7) & ~7;
  }
}

constexpr int kEmitBlock = 128;

// Writes the pairs of enumerated LORs [first, last) at their offsets
// (offsets relative to the chunk start, multiples of 8).  Each lane's
// 8-pair group leaves as two 16-byte key stores and four 16-byte product
// stores into one 32-byte and one 64-byte aligned span, instead of eight
// 4-byte and eight 8-byte stores that each touched 32 lines per warp step.
__global__ void __launch_bounds__(kEmitBlock) k_emit(Grid g, Sino s, Tables t, const float* __restrict__ vals,
                                                     int vals_by_enum, int first, int last,
                                                     const long long* __restrict__ offsets, long long base,
                                                     unsigned sentinel, unsigned* keys, double* prods)
{
  __shared__ unsigned sk[8][kEmitBlock];
  __shared__ double sp[8][kEmitBlock];
  const int tid = threadIdx.x;
  const int i = first + blockIdx.x * kEmitBlock + tid;
  const bool valid = i < last;
  Walk w{};
  bool go = false;
  double v = 0.0;
  long long at = 0;
  if (valid)
  {
    const Lor l = decode_bin(s, i);
    const float fv = vals == nullptr ? 1.0f : __ldg(vals + (vals_by_enum ? i : l.bin));
    v = (double)fv;
    at = offsets[i] - base;
    if (fv != 0.0f)
    {
      double e[6];
      lor_ends(s, t, l, e);
      go = siddon_setup(g, e, w);
    }
  }
  int slot = 0;
  auto flush = [&]() {
    uint4* kd = reinterpret_cast<uint4*>(keys + at);
    kd[0] = make_uint4(sk[0][tid], sk[1][tid], sk[2][tid], sk[3][tid]);
    kd[1] = make_uint4(sk[4][tid], sk[5][tid], sk[6][tid], sk[7][tid]);
    double2* pd = reinterpret_cast<double2*>(prods + at);
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
      pd[q] = make_double2(sp[2 * q][tid], sp[2 * q + 1][tid]);
    }
    at += 8;
  };
  siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      sk[slot][tid] = (unsigned)c;
      sp[slot][tid] = dmul(len, v);
      if (++slot == 8)
      {
        flush();
        slot = 0;
      }
    }
  });
  if (slot > 0)
  {
    for (int q = slot; q < 8; ++q)
    {
      sk[q][tid] = sentinel;
      sp[q][tid] = 0.0;
    }
    flush();
  }
}

// One thread per run of equal voxel (run r: voxel[r], products [start[r],
// start[r] + len[r]) of the sorted array) replays FIR's sequential
// accumulation float(double(acc) + product) in run order.  Neighbouring
// threads take neighbouring voxels, whose runs have similar lengths, and each
// streams its own contiguous run through L1.  (A warp per run, every lane
// replaying the run through shuffles, spent 32 lanes' worth of conversions
// per product and was bound by the conversion pipe: 8.4 ms against this.)
__global__ void __launch_bounds__(256) k_reduce_runs(const int* __restrict__ n_runs, const unsigned* __restrict__ voxel,
                                                     const int* __restrict__ start, const int* __restrict__ len,
                                                     const double* __restrict__ prods, unsigned n_vox, float* img)
{
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= *n_runs)
  {
    return;
  }
  const unsigned v = voxel[r];
  if (v >= n_vox)
  {
    return;  // the padding run
  }
  const double* p = prods + start[r];
  const int n = len[r];
  float acc = img[v];
#pragma unroll 4
  for (int k = 0; k < n; ++k)
  {
    acc = __double2float_rn(dadd((double)acc, __ldg(p + k)));
  }
  img[v] = acc;
}

// The ratio of one OSEM sub-iteration per enumerated LOR
// (reconAlgos.cc:119-158): measured / (projection + bias) when that exceeds
// 1e-5, else 0; with multiplicative factors m, m * measured / (m * projection
// + bias).
//
// With counts, the kernel also writes what k_count would for the ratio: the
// LOR's element count rounded up to a multiple of 8, 0 where the ratio is 0
// (its walk is the one the backprojection will take).
__global__ void __launch_bounds__(256) k_ratio(Grid g, Sino s, Tables t, const double* __restrict__ img,
                                               const float* __restrict__ sino, const float* __restrict__ mult,
                                               const float* __restrict__ bias, float* ratio, int* counts,
                                               int* check)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < s.n_enum;
  Lor l{};
  Walk w{};
  bool go = false;
  if (valid)
  {
    l = decode_bin(s, i);
    double e[6];
    lor_ends(s, t, l, e);
    go = siddon_setup(g, e, w);
  }
  float line = 0.0f;
  int k = 0;
  const bool ok = siddon_walk(g, w, go, [&](bool inside, int c, double len) {
    if (inside)
    {
      line = accumulate(line, len, __ldg(img + c));
      ++k;
    }
  });
  if (!ok && check != nullptr)
  {
    atomicOr(check, kCheckWalkGuard);
  }
  if (valid)
  {
    const float m = mult != nullptr ? __ldg(mult + l.bin) : 1.0f;
    if (mult != nullptr)
    {
      line = __fmul_rn(line, m);
    }
    if (bias != nullptr)
    {
      line = __fadd_rn(line, __ldg(bias + l.bin));
    }
    float q = (go && ok && (double)line > kEps) ? __fdiv_rn(__ldg(sino + l.bin), line) : 0.0f;
    if (mult != nullptr)
    {
      q = __fmul_rn(q, m);
    }
    ratio[i] = q;
    if (counts != nullptr)
    {
      counts[i] = q != 0.0f ? (k + 7) & ~7 : 0;
    }
  }
}

// Greedy chunks of whole LORs: chunk k is [b_k, b_k+1), with b_k+1 the
// largest index whose offset stays within max_pairs of b_k's (at least
// b_k + 1).  max_pairs = min(total, cap), at least floor_pairs.  out: total,
// max_pairs, the number of chunks K, unused, then the (index, offset) of
// b_0 .. b_K.  One thread: a binary search per chunk, so that the host reads
// a few numbers instead of every LOR's offset.
__global__ void k_chunks(const long long* __restrict__ offsets, const int* __restrict__ counts, long long n,
                         long long cap, long long floor_pairs, long long* out)
{
  if (blockIdx.x != 0 || threadIdx.x != 0)
  {
    return;
  }
  const long long total = offsets[n - 1] + counts[n - 1];
  long long mp = total < cap ? total : cap;
  mp = mp < floor_pairs ? floor_pairs : mp;
  auto off = [&](long long i) { return i < n ? offsets[i] : total; };
  long long first = 0, k = 0;
  out[4] = 0;
  out[5] = 0;
  while (first < n)
  {
    const long long limit = off(first) + mp;
    long long lo = first + 1, hi = n;
    if (off(lo) <= limit)
    {
      while (lo < hi)
      {
        const long long mid = (lo + hi + 1) >> 1;
        if (off(mid) <= limit)
          lo = mid;
        else
          hi = mid - 1;
      }
    }
    first = lo;
    ++k;
    out[4 + 2 * k] = first;
    out[5 + 2 * k] = off(first);
  }
  out[0] = total;
  out[1] = mp;
  out[2] = k;
  out[3] = 0;
}

// 64-bit sum of pair counts, for the offsets scan.
struct PairSum
{
  __host__ __device__ long long operator()(long long a, long long b) const { return a + b; }
};

int bits_for(long long n)
{
  int b = 1;
  while ((1LL << b) < n)
  {
    ++b;
  }
  return b;
}

unsigned blocks_for(long long n, int block)
{
  return (unsigned)((n + block - 1) / block);
}
}  // namespace

void launch_ratio(const Grid& g, const Sino& s, const Tables& t, const double* img, const float* sino,
                  const float* mult, const float* bias, float* ratio, int* counts, const LaunchCfg& cfg)
{
  if (s.n_enum > 0)
  {
    k_ratio<<<blocks_for(s.n_enum, cfg.block), cfg.block, 0, cfg.stream>>>(g, s, t, img, sino, mult, bias, ratio,
                                                                          counts, cfg.check);
  }
}

namespace
{
size_t round256(size_t b) { return (b + 255) / 256 * 256; }
}  // namespace

cudaError_t deterministic_backproject(const Grid& g, const Sino& s, const Tables& t, const float* vals,
                                      bool vals_by_enum, const int* counts_in, float* img, const ScratchFn& scratch,
                                      long long max_pairs_cap, long long n_vox, const LaunchCfg& cfg,
                                      long long* launches)
{
  const long long n = s.n_enum;
  if (n == 0)
  {
    return cudaSuccess;
  }
  // 1. path element count of every LOR and their exclusive prefix sum
  size_t scan_bytes = 0;
  // offsets exceed 2^31 pairs on large subsets: the scan must accumulate in
  // 64 bits (ExclusiveSum would accumulate in the counts' int type)
  cudaError_t e = cub::DeviceScan::ExclusiveScan(nullptr, scan_bytes, (const int*)nullptr, (long long*)nullptr,
                                                 PairSum{}, 0LL, (int)n, cfg.stream);
  if (e != cudaSuccess)
  {
    return e;
  }
  // chunk table: 4 header words and (index, offset) of up to n + 1 bounds
  const size_t chunk_words = 4 + 2 * ((size_t)n + 1);
  unsigned char* idx = static_cast<unsigned char*>(scratch(0, round256((size_t)n * 4) + round256((size_t)n * 8) +
                                                                 round256(scan_bytes) + round256(chunk_words * 8)));
  if (idx == nullptr)
  {
    return cudaErrorMemoryAllocation;
  }
  int* counts = reinterpret_cast<int*>(idx);
  const int* cnt = counts_in != nullptr ? counts_in : counts;
  long long* offsets = reinterpret_cast<long long*>(idx + round256((size_t)n * 4));
  void* scan_tmp = idx + round256((size_t)n * 4) + round256((size_t)n * 8);
  long long* chunk_dev =
    reinterpret_cast<long long*>(idx + round256((size_t)n * 4) + round256((size_t)n * 8) + round256(scan_bytes));
  if (counts_in == nullptr)
  {
    k_count<<<blocks_for(n, cfg.block), cfg.block, 0, cfg.stream>>>(g, s, t, vals, vals_by_enum ? 1 : 0, counts,
                                                                    cfg.check);
    *launches += 1;
  }
  e = cub::DeviceScan::ExclusiveScan(scan_tmp, scan_bytes, cnt, offsets, PairSum{}, 0LL, (int)n, cfg.stream);
  if (e == cudaSuccess)
  {
    k_chunks<<<1, 32, 0, cfg.stream>>>(offsets, cnt, n, max_pairs_cap, (long long)g.guard + 8, chunk_dev);
    e = cudaGetLastError();
  }
  // the header and the first bounds in one read; the rest, if there are more
  constexpr size_t kFirstWords = 4 + 2 * 64;
  std::vector<long long> chunk(std::min(chunk_words, kFirstWords));
  if (e == cudaSuccess)
  {
    e = cudaMemcpyAsync(chunk.data(), chunk_dev, chunk.size() * 8, cudaMemcpyDeviceToHost, cfg.stream);
  }
  if (e == cudaSuccess)
  {
    e = cudaStreamSynchronize(cfg.stream);
  }
  if (e != cudaSuccess)
  {
    return e;
  }
  *launches += 2;
  const long long total = chunk[0];
  if (total == 0)
  {
    return cudaGetLastError();
  }
  const size_t used_words = 4 + 2 * ((size_t)chunk[2] + 1);
  if (used_words > chunk.size())
  {
    chunk.resize(used_words);
    e = cudaMemcpyAsync(chunk.data() + kFirstWords, chunk_dev + kFirstWords, (used_words - kFirstWords) * 8,
                        cudaMemcpyDeviceToHost, cfg.stream);
    if (e == cudaSuccess)
    {
      e = cudaStreamSynchronize(cfg.stream);
    }
    if (e != cudaSuccess)
    {
      return e;
    }
  }

  // 2. pair buffers for chunks of at most max_pairs (at least one LOR's
  // padded path)
  const long long max_pairs = chunk[1];
  // runs of one chunk: at most one per voxel, the padding run, and one per pair
  const long long max_runs = max_pairs < n_vox + 1 ? max_pairs : n_vox + 1;
  size_t sort_bytes = 0, rle_bytes = 0, run_scan_bytes = 0;
  e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const unsigned*)nullptr, (unsigned*)nullptr,
                                      (const double*)nullptr, (double*)nullptr, (int)max_pairs, 0, 32, cfg.stream);
  if (e == cudaSuccess)
  {
    e = cub::DeviceRunLengthEncode::Encode(nullptr, rle_bytes, (const unsigned*)nullptr, (unsigned*)nullptr,
                                           (int*)nullptr, (int*)nullptr, (int)max_pairs, cfg.stream);
  }
  if (e == cudaSuccess)
  {
    e = cub::DeviceScan::ExclusiveSum(nullptr, run_scan_bytes, (const int*)nullptr, (int*)nullptr, (int)max_runs,
                                      cfg.stream);
  }
  if (e != cudaSuccess)
  {
    return e;
  }
  const size_t tmp_bytes = std::max(sort_bytes, std::max(rle_bytes, run_scan_bytes));
  const size_t kslab = round256((size_t)max_pairs * 4);
  const size_t pslab = round256((size_t)max_pairs * 8);
  const size_t rslab = round256((size_t)max_runs * 4);
  unsigned char* pb = static_cast<unsigned char*>(
    scratch(1, 2 * kslab + 2 * pslab + 3 * rslab + 256 + round256(tmp_bytes)));
  if (pb == nullptr)
  {
    return cudaErrorMemoryAllocation;
  }
  auto* keys_a = reinterpret_cast<unsigned*>(pb);
  auto* keys_b = reinterpret_cast<unsigned*>(pb + kslab);
  auto* prods_a = reinterpret_cast<double*>(pb + 2 * kslab);
  auto* prods_b = reinterpret_cast<double*>(pb + 2 * kslab + pslab);
  auto* run_voxel = reinterpret_cast<unsigned*>(pb + 2 * kslab + 2 * pslab);
  auto* run_len = reinterpret_cast<int*>(pb + 2 * kslab + 2 * pslab + rslab);
  auto* run_start = reinterpret_cast<int*>(pb + 2 * kslab + 2 * pslab + 2 * rslab);
  auto* n_runs = reinterpret_cast<int*>(pb + 2 * kslab + 2 * pslab + 3 * rslab);
  void* sort_tmp = pb + 2 * kslab + 2 * pslab + 3 * rslab + 256;

  // 3. chunks of whole LORs, reduced in order
  const int key_bits = bits_for(n_vox + 1);  // the padding key n_vox included
  for (long long c = 0; c < chunk[2]; ++c)
  {
    const long long first = chunk[(size_t)(4 + 2 * c)], last = chunk[(size_t)(6 + 2 * c)];
    const long long base = chunk[(size_t)(5 + 2 * c)];
    const long long m = chunk[(size_t)(7 + 2 * c)] - base;
    if (m > 0)
    {
      k_emit<<<blocks_for(last - first, kEmitBlock), kEmitBlock, 0, cfg.stream>>>(
        g, s, t, vals, vals_by_enum ? 1 : 0, (int)first, (int)last, offsets, base, (unsigned)n_vox, keys_a, prods_a);
      size_t tmp = tmp_bytes;
      e = cub::DeviceRadixSort::SortPairs(sort_tmp, tmp, keys_a, keys_b, prods_a, prods_b, (int)m, 0, key_bits,
                                          cfg.stream);
      if (e == cudaSuccess)
      {
        tmp = tmp_bytes;
        e = cub::DeviceRunLengthEncode::Encode(sort_tmp, tmp, keys_b, run_voxel, run_len, n_runs, (int)m, cfg.stream);
      }
      const long long runs_cap = m < max_runs ? m : max_runs;
      if (e == cudaSuccess)
      {
        // run starts: exclusive sum of the lengths (entries past the run
        // count are never read)
        tmp = tmp_bytes;
        e = cub::DeviceScan::ExclusiveSum(sort_tmp, tmp, run_len, run_start, (int)runs_cap, cfg.stream);
      }
      if (e != cudaSuccess)
      {
        return e;
      }
      k_reduce_runs<<<blocks_for(runs_cap, 256), 256, 0, cfg.stream>>>(n_runs, run_voxel, run_start, run_len,
                                                                      prods_b, (unsigned)n_vox, img);
      *launches += 2;
    }
  }
  return cudaGetLastError();
}
}  // namespace fir
