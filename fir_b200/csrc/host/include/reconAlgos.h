// FIR's reconstruction entry points (src_lib/reconAlgos.h:9-45), same
// signatures; the OSEM loop runs on the GPU (fir_osem).
#pragma once

#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>

#include <optional>
#include <string>
#include <vector>

struct OSEMCoreParams
{
  int nIterations{1};
  int nSubsets{1};
  int saveInterval{0};
  float cutRadius{0.0};
  int convolutionInterval{0};
  std::vector<float> fwhmXYZ{0.0, 0.0, 0.0};
};

namespace reconAlgos
{
// OSEM with FIR's update, gates, filter and cut (reconAlgos.cc:63-201).
// Intermediate images every saveInterval sub-iterations are written to
// <outputVolFileName>_subiter_<k>.
void OSEM(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol,
          const std::string& outputVolFileName, const OSEMCoreParams& params, const VolData& sensitivityMap,
          const std::optional<ProjData>& biasProj);

// FIR's resolution-modelling OSEM variant, with FIR's order of operations
// (reconAlgos.cc:203-367); sensitivityMap is filtered in place.
void OSEM_ResoReco(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol,
                   const std::string& outputVolFileName, const OSEMCoreParams& params, VolData& sensitivityMap,
                   const std::optional<ProjData>& biasProj);
}  // namespace reconAlgos
