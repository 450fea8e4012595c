// Test infrastructure only (part of the oracle): an extern "C" harness that
// drives the unmodified FIR library through its own public C++ API, so that
// Python tests and the CPU-baseline leg of bench.py can call it with ctypes.
// It is compiled together with FIR's sources by oracle/Makefile into
// oracle/_ref/libfirref.so.  Every entry point returns 0 on success and -1 on
// a FIR exception (message in ref_last_error()).
//
// FIR entry points driven here (paths inside the FIR project):
//   Siddon::computePath            src_lib/Siddon.cc:112-258
//   projections::forward/backward  src_lib/projections.cc:15-184
//   projections::computeSensitivityVol  src_lib/projections.cc:186-197
//   reconAlgos::OSEM               src_lib/reconAlgos.cc:63-201
//   operations::*                  src_lib/operations.cc:11-284
//   ProjData::exponential, *=      src_lib/ProjData.cc:481-539
//   ProjData::getCrystal*Coord     src_lib/ProjData.cc:198-340
//   ScannerData position tables    src_lib/ScannerData.cc:248-377

#include <ProjData.h>
#include <ScannerData.h>
#include <Siddon.h>
#include <VolData.h>
#include <operations.h>
#include <projections.h>
#include <reconAlgos.h>

#include <cstring>
#include <iostream>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
thread_local std::string g_lastError;

struct Quiet
{
  // FIR prints progress to stdout; keep test and bench output clean.
  std::stringstream sink;
  std::streambuf* saved;
  Quiet(): saved{std::cout.rdbuf(sink.rdbuf())} {}
  ~Quiet() { std::cout.rdbuf(saved); }
};

template<typename F>
int guarded(F&& f)
{
  try
  {
    Quiet q;
    f();
    return 0;
  }
  catch (const std::exception& ex)
  {
    g_lastError = ex.what();
    return -1;
  }
}
}

extern "C" {

struct ref_vol
{
  int nx, ny, nz;
  double vx, vy, vz;
  double ox, oy, oz;
  int nframes;
};

const char* ref_last_error() { return g_lastError.c_str(); }

void ref_set_threads(int n)
{
#ifdef _OPENMP
  if (n > 0)
  {
    omp_set_num_threads(n);
  }
#else
  (void)n;
#endif
}

int ref_get_threads()
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}

namespace
{
VolHeader toHeader(const ref_vol* v, int nframes)
{
  VolHeader h;
  h.setDefaults();
  h.volSize = {v->nx, v->ny, v->nz};
  h.voxelExtent = {v->vx, v->vy, v->vz};
  h.volOffset = {v->ox, v->oy, v->oz};
  h.nFrames = nframes;
  return h;
}

void copyIn(VolData& vol, const float* src)
{
  const auto n = static_cast<size_t>(vol.getNVoxelsPerFrame()) * vol.getNFrames();
  vol.setActiveFrame(0);
  std::memcpy(vol.getDataArray(), src, n * sizeof(float));
}

void copyOut(const VolData& vol, float* dst)
{
  const auto n = static_cast<size_t>(vol.getNVoxelsPerFrame()) * vol.getNFrames();
  vol.setActiveFrame(0);
  std::memcpy(dst, vol.getDataArray(), n * sizeof(float));
}

size_t segBins(const ProjData& p, int seg)
{
  const auto& g = p.getGeometry();
  return static_cast<size_t>(g.getNAxialCoords(seg)) * g.nViews *
         p.getHeader().nTangCoords;
}

void projIn(ProjData& p, const float* src)
{
  const auto& g = p.getGeometry();
  size_t off = 0;
  for (int seg = -g.segOffset; seg <= g.segOffset; ++seg)
  {
    const auto n = segBins(p, seg);
    std::memcpy(p.getDataArray()[seg + g.segOffset], src + off, n * sizeof(float));
    off += n;
  }
}

void projOut(const ProjData& p, float* dst)
{
  const auto& g = p.getGeometry();
  size_t off = 0;
  for (int seg = -g.segOffset; seg <= g.segOffset; ++seg)
  {
    const auto n = segBins(p, seg);
    std::memcpy(dst + off, p.getDataArray()[seg + g.segOffset], n * sizeof(float));
    off += n;
  }
}
}

extern "C" {

// Per-LOR Siddon paths for n segments given by their end points
// pts[6*i .. 6*i+5] = (x1, y1, z1, x2, y2, z2).  Output row i holds up to cap
// elements; counts[i] = emitted elements, crosses[i] = return value.
int ref_siddon_paths(
  const ref_vol* v,
  int n,
  const double* pts,
  int cap,
  int* coords,
  double* lengths,
  int* counts,
  int* crosses)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, 1));
      Siddon siddon(vol);
      const int maxLen = v->nx + v->ny + v->nz + 2;
      std::vector<types::PathElement> path(maxLen);
      for (int i = 0; i < n; ++i)
      {
        const double* p = pts + 6 * static_cast<size_t>(i);
        crosses[i] = siddon.computePath(p[0], p[1], p[2], p[3], p[4], p[5], path.data());
        int k = 0;
        for (; path[k].coord != -1; ++k)
        {
          if (k < cap)
          {
            coords[static_cast<size_t>(i) * cap + k] = path[k].coord;
            lengths[static_cast<size_t>(i) * cap + k] = path[k].length;
          }
        }
        counts[i] = k;
      }
    });
}

int ref_scanner_tables(
  const char* scannerFile,
  int* nRings,
  int* nCrystalsPerRing,
  double* xy,
  double* z,
  int capCrystals,
  int capSlices)
{
  return guarded(
    [&]
    {
      ScannerData scanner(scannerFile);
      // The tables are only reachable through the path-tracing accessors.
      const auto* t = scanner.getCrystalXYPositionVector();
      const auto* s = scanner.getSliceZPositionVector();
      for (int i = 0; i < capCrystals; ++i)
      {
        xy[2 * i] = t[i].x;
        xy[2 * i + 1] = t[i].y;
      }
      for (int i = 0; i < capSlices; ++i)
      {
        z[i] = s[i];
      }
      (void)nRings;
      (void)nCrystalsPerRing;
    });
}

// Number of path elements FIR's Siddon emits for every bin (file order),
// using FIR's own traversal (computePathBetweenCrystals) on all threads.
int ref_path_counts(
  const char* scannerFile,
  const char* projHeader,
  const ref_vol* v,
  int* counts)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      ScannerData scanner(scannerFile);
      VolData vol(toHeader(v, 1));
      Siddon siddon(vol);
      const auto& g = proj.getGeometry();
      const auto nTang = proj.getHeader().nTangCoords;
      size_t base = 0;
      for (int seg = -g.segOffset; seg <= g.segOffset; ++seg)
      {
        const int nax = g.getNAxialCoords(seg);
        const size_t bpv = static_cast<size_t>(nax) * nTang;
#pragma omp parallel for schedule(dynamic, 1)
        for (int view = 0; view < g.nViews; ++view)
        {
          auto* path = siddon.getThreadLocalPathElements();
          size_t b = base + view * bpv;
          for (int ax = 0; ax < nax; ++ax)
          {
            const auto [a1, a2] = proj.getCrystalAxialCoord(seg, ax);
            for (int t = -g.tangCoordOffset; t < -g.tangCoordOffset + nTang; ++t)
            {
              const auto [c1, c2] = proj.getCrystalAngCoord(view, t);
              siddon.computePathBetweenCrystals(scanner, a1, c1, a2, c2, path);
              int k = 0;
              while (path[k].coord != -1)
              {
                ++k;
              }
              counts[b++] = k;
            }
          }
        }
        base += bpv * g.nViews;
      }
    });
}

// out[0..6] = nBins, segOffset, tangCoordOffset, nViews, halfSegmentSpan,
// maxRingDiff, nTangCoords (after check()); out[7..] = nAxialCoords.
int ref_proj_geometry(const char* projHeader, int* out, int cap)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      const auto& g = proj.getGeometry();
      out[0] = g.nBins;
      out[1] = g.segOffset;
      out[2] = g.tangCoordOffset;
      out[3] = g.nViews;
      out[4] = g.halfSegmentSpan;
      out[5] = g.maxRingDiff;
      out[6] = proj.getHeader().nTangCoords;
      for (int i = 0; i < static_cast<int>(g.nAxialCoords.size()) && 7 + i < cap; ++i)
      {
        out[7 + i] = g.nAxialCoords[i];
      }
    });
}

// Crystal pair of every bin, flat file order: out[4*b..] = (axial1, ang1,
// axial2, ang2).
int ref_lor_table(const char* projHeader, int* out)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      const auto& g = proj.getGeometry();
      const auto nTang = proj.getHeader().nTangCoords;
      size_t b = 0;
      for (int seg = -g.segOffset; seg <= g.segOffset; ++seg)
        for (int view = 0; view < g.nViews; ++view)
          for (int ax = 0; ax < g.getNAxialCoords(seg); ++ax)
            for (int t = -g.tangCoordOffset; t < -g.tangCoordOffset + nTang; ++t)
            {
              const auto [a1, a2] = proj.getCrystalAxialCoord(seg, ax);
              const auto [c1, c2] = proj.getCrystalAngCoord(view, t);
              out[4 * b] = a1;
              out[4 * b + 1] = c1;
              out[4 * b + 2] = a2;
              out[4 * b + 3] = c2;
              ++b;
            }
    });
}

int ref_forward(
  const char* scannerFile,
  const char* projHeader,
  const ref_vol* v,
  const float* img,
  float* sino)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      ScannerData scanner(scannerFile);
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projections::forward(vol, scanner, proj);
      projOut(proj, sino);
    });
}

int ref_backward(
  const char* scannerFile,
  const char* projHeader,
  const float* sino,
  const ref_vol* v,
  int nSubsets,
  float* img)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(proj, sino);
      ScannerData scanner(scannerFile);
      VolData vol(toHeader(v, nSubsets));
      projections::backward(proj, scanner, vol, nSubsets);
      copyOut(vol, img);
    });
}

int ref_sensitivity(
  const char* scannerFile,
  const char* projHeader,
  const ref_vol* v,
  int nSubsets,
  float* sens)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      ScannerData scanner(scannerFile);
      VolData vol(toHeader(v, nSubsets));
      projections::computeSensitivityVol(proj, scanner, vol, nSubsets);
      copyOut(vol, sens);
    });
}

// reconAlgos::OSEM on an image that already holds the initial estimate.
// sens holds nSubsets frames.  outName is only used when saveInterval > 0.
int ref_osem(
  const char* scannerFile,
  const char* projHeader,
  const float* sino,
  const float* bias,
  const ref_vol* v,
  float* img,
  const float* sens,
  int nIterations,
  int nSubsets,
  float cutRadius,
  int convolutionInterval,
  const float* fwhmXYZ,
  int saveInterval,
  const char* outName)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(proj, sino);
      std::optional<ProjData> biasProj;
      if (bias != nullptr)
      {
        biasProj.emplace(proj, ProjData::ConstructionMode::ALLOCATE);
        projIn(*biasProj, bias);
      }
      ScannerData scanner(scannerFile);
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      VolData sensVol(toHeader(v, nSubsets));
      copyIn(sensVol, sens);
      OSEMCoreParams params;
      params.nIterations = nIterations;
      params.nSubsets = nSubsets;
      params.saveInterval = saveInterval;
      params.cutRadius = cutRadius;
      params.convolutionInterval = convolutionInterval;
      params.fwhmXYZ = {fwhmXYZ[0], fwhmXYZ[1], fwhmXYZ[2]};
      reconAlgos::OSEM(
        proj,
        scanner,
        vol,
        outName ? std::string(outName) : std::string("osem"),
        params,
        sensVol,
        biasProj);
      copyOut(vol, img);
    });
}

// reconAlgos::OSEM_ResoReco (reconAlgos.cc:203-367) on FIR's own code; the
// sensitivity volume of nSensFrames frames is copied back (FIR filters it in
// place).
int ref_osem_reso_reco(
  const char* scannerFile,
  const char* projHeader,
  const float* sino,
  const float* bias,
  const ref_vol* v,
  float* img,
  float* sens,
  int nSensFrames,
  int nIterations,
  int nSubsets,
  float cutRadius,
  int convolutionInterval,
  const float* fwhmXYZ,
  const char* outName)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(proj, sino);
      std::optional<ProjData> biasProj;
      if (bias != nullptr)
      {
        biasProj.emplace(proj, ProjData::ConstructionMode::ALLOCATE);
        projIn(*biasProj, bias);
      }
      ScannerData scanner(scannerFile);
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      VolData sensVol(toHeader(v, nSensFrames));
      copyIn(sensVol, sens);
      OSEMCoreParams params;
      params.nIterations = nIterations;
      params.nSubsets = nSubsets;
      params.saveInterval = 0;
      params.cutRadius = cutRadius;
      params.convolutionInterval = convolutionInterval;
      params.fwhmXYZ = {fwhmXYZ[0], fwhmXYZ[1], fwhmXYZ[2]};
      reconAlgos::OSEM_ResoReco(
        proj,
        scanner,
        vol,
        outName ? std::string(outName) : std::string("osem_reso"),
        params,
        sensVol,
        biasProj);
      copyOut(vol, img);
      copyOut(sensVol, sens);
    });
}

int ref_convolve(const ref_vol* v, float* img, const float* fwhmXYZ, float cutRadius)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, v->nframes > 0 ? v->nframes : 1));
      copyIn(vol, img);
      operations::convolve(vol, {fwhmXYZ[0], fwhmXYZ[1], fwhmXYZ[2]}, cutRadius);
      copyOut(vol, img);
    });
}

int ref_cut_circle(const ref_vol* v, float* img, float cutRadius)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      operations::cutCircle(vol, cutRadius);
      copyOut(vol, img);
    });
}

int ref_apply_mask(const ref_vol* v, float* img, const float* mask)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      VolData maskVol(toHeader(v, 1));
      copyIn(maskVol, mask);
      operations::applyMask(vol, maskVol);
      copyOut(vol, img);
    });
}

int ref_hu_to_mu(const ref_vol* v, float* img)
{
  return guarded(
    [&]
    {
      VolData vol(toHeader(v, 1));
      copyIn(vol, img);
      operations::HounsfieldToMuMap(vol);
      copyOut(vol, img);
    });
}

int ref_proj_exponential(const char* projHeader, float* sino)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(proj, sino);
      proj.exponential();
      projOut(proj, sino);
    });
}

int ref_proj_multiply(const char* projHeader, float* a, const float* b)
{
  return guarded(
    [&]
    {
      ProjData pa(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(pa, a);
      ProjData pb(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(pb, b);
      pa *= pb;
      projOut(pa, a);
    });
}

// ProjData::getBinCoordinates (ProjData.cc:342-479) on n crystal pairs
// (ring1, crystal1, ring2, crystal2): out[5i] = returned flag, then seg,
// view, axial, tang (0 where FIR returns false).
int ref_bin_coordinates(const char* projHeader, long long n, const int* pairs, int* out)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      for (long long i = 0; i < n; ++i)
      {
        int seg = 0, view = 0, axial = 0, tang = 0;
        const bool ok =
          proj.getBinCoordinates(pairs[4 * i], pairs[4 * i + 1], pairs[4 * i + 2], pairs[4 * i + 3], &seg, &view,
                                 &axial, &tang);
        out[5 * i] = ok ? 1 : 0;
        out[5 * i + 1] = ok ? seg : 0;
        out[5 * i + 2] = ok ? view : 0;
        out[5 * i + 3] = ok ? axial : 0;
        out[5 * i + 4] = ok ? tang : 0;
      }
    });
}

// ProjData::rebinWeight (ProjData.cc:541-615) applied to sino in place.
int ref_rebin_weight(const char* projHeader, float* sino)
{
  return guarded(
    [&]
    {
      ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
      projIn(proj, sino);
      proj.rebinWeight();
      projOut(proj, sino);
    });
}

// Element-wise EM image update of reconAlgos.cc:161-166, via VolData's own
// operators (VolData.cc:305-343): bp /= sens; img *= bp.
int ref_em_update(const ref_vol* v, float* img, float* bp, const float* sens)
{
  return guarded(
    [&]
    {
      VolData x(toHeader(v, 1));
      copyIn(x, img);
      VolData b(toHeader(v, 1));
      copyIn(b, bp);
      VolData s(toHeader(v, 1));
      copyIn(s, sens);
      b /= s;
      x *= b;
      copyOut(x, img);
      copyOut(b, bp);
    });
}

}
