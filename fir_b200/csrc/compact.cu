// The non-zero bins of a subset as a compacted enumeration (Sino::list), for
// FIR_OPT_SKIP_ZERO_BINS.  A bin whose measured value is 0 has a ratio of
// exactly 0 in reconAlgos.cc:152-157, so its backprojection adds nothing and
// skipping it is exact.  Skipped inside the fused kernel, such a bin still
// holds its lane while the other lanes of the warp trace; listed out, the
// remaining LORs fill whole warps.  The list keeps the enumeration order, so
// neighbouring lanes still trace neighbouring LORs.
//
// One kernel writes a byte flag per enumerated index (the Sino stays a kernel
// parameter), then CUB's flagged selection over the counting sequence writes
// the list.  A predicate functor holding the Sino (about 3 KB) was copied per
// thread by the selection kernel and took about 1 ms per clinical subset.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "internal.h"

namespace fir
{
namespace
{
__global__ void __launch_bounds__(256) k_nonzero_flags(Sino s, const float* __restrict__ sino,
                                                       unsigned char* __restrict__ flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < s.n_enum)
  {
    flags[i] = __ldg(sino + decode_bin(s, i).bin) != 0.0f ? 1 : 0;
  }
}
}  // namespace

cudaError_t launch_nonzero_list(const Sino& s, const float* sino, int* list, int* count, void* temp,
                                size_t* temp_bytes, const LaunchCfg& cfg)
{
  // temp: the flags (n_enum bytes, rounded to 256) then CUB's scratch
  const size_t flag_bytes = ((size_t)s.n_enum + 255) / 256 * 256;
  size_t cub_bytes = 0;
  unsigned char* flags = static_cast<unsigned char*>(temp);
  cudaError_t e = cub::DeviceSelect::Flagged(nullptr, cub_bytes, thrust::counting_iterator<int>(0),
                                             (const unsigned char*)nullptr, (int*)nullptr, (int*)nullptr, s.n_enum,
                                             cfg.stream);
  if (e != cudaSuccess || temp == nullptr)
  {
    *temp_bytes = flag_bytes + cub_bytes;
    return e;
  }
  Sino plain = s;
  plain.list = nullptr;
  plain.list_n = nullptr;
  k_nonzero_flags<<<(unsigned)((s.n_enum + 255) / 256), 256, 0, cfg.stream>>>(plain, sino, flags);
  e = cudaGetLastError();
  if (e != cudaSuccess)
  {
    return e;
  }
  return cub::DeviceSelect::Flagged(flags + flag_bytes, cub_bytes, thrust::counting_iterator<int>(0), flags, list,
                                    count, s.n_enum, cfg.stream);
}
}  // namespace fir
