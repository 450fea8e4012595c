// Internal interface of the C ABI's host code, shared by capi.cu and
// capi_batch.cu: failures and their statuses, validation of FIR's headers,
// device buffers, and the context.  Not installed; not part of the ABI.
#pragma once

#include "../../include/fir_cuda.h"
#include "internal.h"

#include <nvtx3/nvToolsExt.h>

#include <exception>
#include <new>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace fir::abi
{
// The thread-local message of the last failed call (fir_last_error).
extern thread_local std::string g_error;

struct Failure
{
  fir_status status;
  std::string message;
};

template<typename... Args>
[[noreturn]] void fail(fir_status s, Args&&... args)
{
  std::ostringstream os;
  (os << ... << args);
  throw Failure{s, os.str()};
}

// Throws a Failure with the CUDA error's text when e is not cudaSuccess.
void cuda_ok(cudaError_t e, const char* what);

// An NVTX range named after the ABI function brackets every call, so that
// profilers show the host-side structure around the kernels.
struct NvtxRange
{
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

template<typename F>
fir_status guarded(const char* name, F&& f)
{
  const NvtxRange range(name);
  try
  {
    f();
    return FIR_OK;
  }
  catch (const Failure& x)
  {
    g_error = x.message;
    return x.status;
  }
  catch (const std::bad_alloc&)
  {
    g_error = "host allocation failed";
    return FIR_ERR_OUT_OF_MEMORY;
  }
  catch (const std::exception& x)
  {
    g_error = x.what();
    return FIR_ERR_INVALID_ARGUMENT;
  }
}

// ------------------------------------------------------------ validation

struct ProjInfo
{
  fir_proj_desc d;
  fir_proj_info g;
  std::vector<int> n_axial;
};
// ProjHeader::check + ProjGeometry::fill, with FIR's messages.
ProjInfo check_proj(const fir_proj_desc* desc);

struct ScannerInfo
{
  int n_rings = 0, n_cpr = 0;
  std::vector<double> xy, z;
};
// ScannerHeader::check + the crystal and slice tables (when tables).
ScannerInfo scanner_tables(const fir_scanner_desc* desc, bool tables);

struct VolInfo
{
  fir_vol_desc d;
  long long nvox;  // per frame
};
VolInfo check_vol(const fir_vol_desc* v);
void check_frames(const VolInfo& v, int n);
void check_subsets(const ProjInfo& p, int n_subsets);
void check_osem_params(const fir_osem_params* prm, const ProjInfo& p);

// ------------------------------------------------------------ buffers

struct DevBuf
{
  void* p = nullptr;
  size_t bytes = 0;

  void* ensure(size_t n)
  {
    if (n > bytes)
    {
      if (p != nullptr)
      {
        cudaFree(p);
        p = nullptr;
        bytes = 0;
      }
      cuda_ok(cudaMalloc(&p, n), "cudaMalloc");
      bytes = n;
    }
    return p;
  }

  void release()
  {
    if (p != nullptr)
    {
      cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
  }
};
}  // namespace fir::abi

// ------------------------------------------------------------ context

struct fir_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  int geometry = FIR_GEOMETRY_REFERENCE;
  int backproj = FIR_BACKPROJ_ATOMIC;
  int skip_zero = 0;
  int block = 128;
  long long det_chunk = 1LL << 28;
  int step_limit = 0;  // FIR_OPT_STEP_LIMIT
  int traversal = FIR_TRAVERSAL_EXACT;  // FIR_OPT_TRAVERSAL
  long long launches = 0;
  long long l2_bytes = 0;  // the device's L2 size, read on first use

  bool have_scanner = false;
  int scan_rings = 0, scan_cpr = 0;
  fir::abi::DevBuf xy, z;

  fir::abi::DevBuf check;     // device check word
  int* check_host = nullptr;  // pinned mirror

  fir::abi::DevBuf bp, conv1, conv2, conv_copy, mu, wide, det, det_pairs, ratio, frames_il, frames_acc, psf_blur, psf_sens, rebin;
  fir::abi::DevBuf wide_t, bp_t;  // x/y-exchanged double image and accumulator of the fused kernel
  fir::abi::DevBuf img_t;         // x/y-exchanged float image (float traversal, float gathers)
  fir::abi::DevBuf compact;       // non-zero bins of a subset (FIR_OPT_SKIP_ZERO_BINS) and CUB scratch
  fir::abi::DevBuf frames_il_t, frames_acc_t;  // the same for the multi-frame projectors
  std::vector<fir::abi::DevBuf> staging;

  // pipelined input of fir_osem from pinned host memory
  std::vector<fir::abi::DevBuf> pipe;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> pipe_events;

  // projector-kernel timing (FIR_OPT_TIMING)
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending;
  double timed_ms = 0.0;
  long long timed_n = 0;
};

namespace fir::abi
{
// Makes the context's device current; fails on NULL.
fir_ctx& check_ctx(fir_ctx* c);
// The traversal grid of a volume under the context's geometry mode.
Grid grid_of(const fir_ctx& c, const VolInfo& v);
// Whether a projector uses x/y-exchanged images for LORs running mostly
// along x: while both orientations of the images it reads and accumulates
// (bytes_per_voxel, both orientations counted; 24 for the fused OSEM
// kernel's double image and float accumulator) fit in L2.
bool use_exchanged(fir_ctx& c, const Grid& g, double bytes_per_voxel = 24.0);
// The enumeration of subset `subset` of n_subsets.
Sino sino_of(const ProjInfo& p, int n_subsets, int subset);
// Reads and clears the device check word; fails when it is set.
void read_checks(fir_ctx& c);
// operations::convolve's taps along one axis.
Taps gauss_taps(float fwhm, double vox, bool double_sigma);
}  // namespace fir::abi
