// GPU context of the C++ drop-in layer (see runtime.h).
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <console.h>
#include <runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

namespace
{
struct Holder
{
  fir_ctx* ctx = nullptr;
  bool haveScanner = false;
  fir_scanner_desc scanner{};
  bool timing = false;
  std::chrono::steady_clock::time_point start;

  ~Holder()
  {
    if (ctx != nullptr)
    {
      fir_ctx_destroy(ctx);
    }
  }
};

thread_local Holder g_holder;
}  // namespace

namespace fir_runtime
{
void check(fir_status status, const char* what)
{
  if (status != FIR_OK)
  {
    error(fir_last_error(), " (", what, ")");
  }
}

fir_ctx* context()
{
  if (g_holder.ctx == nullptr)
  {
    const char* dev = std::getenv("FIR_DEVICE");
    check(fir_ctx_create(&g_holder.ctx, dev ? std::atoi(dev) : 0), "creating the GPU context");
    g_holder.start = std::chrono::steady_clock::now();
    if (const char* t = std::getenv("FIR_TIMING_JSON"))
    {
      if (std::strcmp(t, "0") != 0)
      {
        check(fir_ctx_set_option(g_holder.ctx, FIR_OPT_TIMING, 1), "FIR_TIMING_JSON");
        g_holder.timing = true;
      }
    }
    if (const char* g = std::getenv("FIR_GEOMETRY"))
    {
      if (std::strcmp(g, "exact") == 0)
      {
        check(fir_ctx_set_option(g_holder.ctx, FIR_OPT_GEOMETRY, FIR_GEOMETRY_EXACT), "FIR_GEOMETRY");
      }
    }
  }
  return g_holder.ctx;
}

void reportTiming(const char* program)
{
  if (!g_holder.timing || g_holder.ctx == nullptr)
  {
    return;
  }
  double ms = 0.0;
  long long n = 0;
  check(fir_ctx_projector_time(g_holder.ctx, &ms, &n, 0), "timing");
  const double wall =
    std::chrono::duration<double>(std::chrono::steady_clock::now() - g_holder.start).count();
  std::fprintf(stderr,
               "{\"program\": \"%s\", \"wall_s\": %.6f, \"projector_ms\": %.3f, \"projector_launches\": %lld, "
               "\"kernel_launches\": %lld}\n",
               program, wall, ms, n, fir_ctx_launch_count(g_holder.ctx));
}

void useScanner(const ScannerData& scanner)
{
  const fir_scanner_desc d = scanner.descriptor();
  fir_ctx* c = context();
  if (!g_holder.haveScanner || std::memcmp(&d, &g_holder.scanner, sizeof(d)) != 0)
  {
    check(fir_ctx_set_scanner(c, &d), "scanner");
    g_holder.scanner = d;
    g_holder.haveScanner = true;
  }
}

fir_vol_desc volDesc(const VolData& vol, int nFrames)
{
  const auto& h = vol.getHeader();
  fir_vol_desc d;
  d.nx = h.volSize.nPixelsX;
  d.ny = h.volSize.nPixelsY;
  d.nz = h.volSize.nSlices;
  d.voxel_x = h.voxelExtent.pixelWidth;
  d.voxel_y = h.voxelExtent.pixelHeight;
  d.voxel_z = h.voxelExtent.sliceThickness;
  d.offset_x = h.volOffset.x;
  d.offset_y = h.volOffset.y;
  d.offset_z = h.volOffset.z;
  d.n_frames = nFrames;
  return d;
}

fir_proj_desc projDesc(const ProjData& proj)
{
  const auto& h = proj.getHeader();
  return fir_proj_desc{h.nRings, h.nCrystalsPerRing, h.segmentSpan, h.nSegments, h.nTangCoords};
}
}  // namespace fir_runtime
