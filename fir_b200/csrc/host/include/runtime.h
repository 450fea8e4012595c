// Process-wide GPU context of the C++ drop-in layer.  FIR's C++ entry points
// (projections::, reconAlgos::, operations::, ProjData arithmetic) run through
// the C ABI of include/fir_cuda.h on one fir_ctx per host thread, created on
// first use on the device named by FIR_DEVICE (default 0).  A failing ABI call
// throws std::runtime_error with FIR's "ERROR: ..." text.
#pragma once

#include <fir_cuda.h>

#include <string>

class ScannerData;
class VolData;
class ProjData;

namespace fir_runtime
{
fir_ctx* context();
// Makes the context's scanner tables those of `scanner`.
void useScanner(const ScannerData& scanner);
// Throws on a non-OK status.
void check(fir_status status, const char* what);
// With FIR_TIMING_JSON set (not "0") when the context was created: prints
// one JSON line to stderr with the wall time since then, the device time and
// number of projector launches, and the number of kernel launches.
void reportTiming(const char* program);

fir_vol_desc volDesc(const VolData& vol, int nFrames);
fir_proj_desc projDesc(const ProjData& proj);
}  // namespace fir_runtime
