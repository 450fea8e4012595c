// The non-zero bins of a subset as a compacted enumeration (Sino::list), for
// FIR_OPT_SKIP_ZERO_BINS.  A bin whose measured value is 0 has a ratio of
// exactly 0 in reconAlgos.cc:152-157, so its backprojection adds nothing and
// skipping it is exact.  Skipped inside the fused kernel, such a bin still
// holds its lane while the other lanes of the warp trace; listed out, the
// remaining LORs fill whole warps.  The list keeps the enumeration order, so
// neighbouring lanes still trace neighbouring LORs.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "internal.h"

namespace fir
{
namespace
{
struct NonZeroBin
{
  Sino s;
  const float* sino;

  __device__ __forceinline__ bool operator()(int i) const { return __ldg(sino + decode_bin(s, i).bin) != 0.0f; }
};
}  // namespace

cudaError_t launch_nonzero_list(const Sino& s, const float* sino, int* list, int* count, void* temp,
                                size_t* temp_bytes, const LaunchCfg& cfg)
{
  Sino plain = s;
  plain.list = nullptr;
  plain.list_n = nullptr;
  return cub::DeviceSelect::If(temp, *temp_bytes, thrust::counting_iterator<int>(0), list, count, s.n_enum,
                               NonZeroBin{plain, sino}, cfg.stream);
}
}  // namespace fir
