// reconAlgos:: entry points over the C ABI (FIR: src_lib/reconAlgos.cc).
#include <console.h>
#include <operations.h>
#include <reconAlgos.h>
#include <runtime.h>

#include <algorithm>
#include <cstring>

namespace
{
struct SaveTarget
{
  VolData* vol;
  const std::string* name;
};

// fir_osem_save_fn: writes <name>_subiter_<k> like reconAlgos.cc:189-198
void saveSubiteration(void* user, int subiter, const float* img)
{
  auto* t = static_cast<SaveTarget*>(user);
  float* dst = t->vol->getDataArray();
  std::copy(img, img + t->vol->getNVoxelsPerFrame(), dst);
  t->vol->write(*t->name + "_subiter_" + std::to_string(subiter));
}

fir_osem_params toParams(const OSEMCoreParams& p)
{
  if (p.fwhmXYZ.size() < 3)
  {
    error("convolution FWHM must have three elements");
  }
  fir_osem_params o;
  o.n_iterations = p.nIterations;
  o.n_subsets = p.nSubsets;
  o.save_interval = p.saveInterval;
  o.cut_radius = p.cutRadius;
  o.convolution_interval = p.convolutionInterval;
  for (int i = 0; i < 3; ++i)
  {
    o.fwhm_xyz[i] = p.fwhmXYZ[i];
  }
  return o;
}

void checkSensitivity(const VolData& sens, const VolData& vol, int nSubsets)
{
  if (sens.getNFrames() < nSubsets)
  {
    error("Invalid frame");
  }
  if (sens.getHeader() != vol.getHeader())
  {
    error("Sensitivity volume provided doesn't fit with output volume provided");
  }
}
}  // namespace

namespace reconAlgos
{
void OSEM(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol,
          const std::string& outputVolFileName, const OSEMCoreParams& params, const VolData& sensitivityMap,
          const std::optional<ProjData>& biasProj)
{
  echo("OSEM:");
  scanner.checkProjData(inputProj);
  inputProj.checkNSubsets(params.nSubsets);
  checkSensitivity(sensitivityMap, outputVol, params.nSubsets);
  if (biasProj && !(biasProj->getHeader() == inputProj.getHeader()))
  {
    error("Bias projection doesn't fit with the input projection");
  }
  fir_runtime::useScanner(scanner);
  const fir_osem_params p = toParams(params);
  const fir_vol_desc vd = fir_runtime::volDesc(outputVol, 1);
  const fir_proj_desc pd = fir_runtime::projDesc(inputProj);
  SaveTarget target{&outputVol, &outputVolFileName};
  print("Iterations: ", params.nIterations, ", subsets: ", params.nSubsets);
  fir_runtime::check(fir_osem(fir_runtime::context(), &pd, inputProj.getBins(),
                              biasProj ? biasProj->getBins() : nullptr, &vd, outputVol.getDataArray(),
                              sensitivityMap.getAllFrames(), &p, &saveSubiteration, &target),
                     "OSEM");
  if (params.nIterations > 0)
  {
    sensitivityMap.setActiveFrame(params.nSubsets - 1);
  }
}

// FIR's resolution-modelling variant as FIR runs it (reconAlgos.cc:203-367):
// every frame of the sensitivity volume is filtered once, in place; each
// sub-iteration projects the unfiltered image, filters the backprojection,
// divides the image (not the backprojection) by the subset's sensitivity
// frame and multiplies it by the filtered backprojection.  The whole loop
// runs on the device (fir_osem_reso_reco); the volumes are copied in once
// and out once.
void OSEM_ResoReco(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol,
                   const std::string& outputVolFileName, const OSEMCoreParams& params, VolData& sensitivityMap,
                   const std::optional<ProjData>& biasProj)
{
  echo("OSEM_ResoReco:");
  scanner.checkProjData(inputProj);
  inputProj.checkNSubsets(params.nSubsets);
  checkSensitivity(sensitivityMap, outputVol, params.nSubsets);
  if (biasProj && !(biasProj->getHeader() == inputProj.getHeader()))
  {
    error("Bias projection doesn't fit with the input projection");
  }
  const fir_osem_params p = toParams(params);
  fir_runtime::useScanner(scanner);
  const fir_vol_desc vd = fir_runtime::volDesc(outputVol, 1);
  const fir_proj_desc pd = fir_runtime::projDesc(inputProj);
  SaveTarget target{&outputVol, &outputVolFileName};
  print("Iterations: ", params.nIterations, ", subsets: ", params.nSubsets);
  fir_runtime::check(fir_osem_reso_reco(fir_runtime::context(), &pd, inputProj.getBins(),
                                        biasProj ? biasProj->getBins() : nullptr, &vd, outputVol.getDataArray(),
                                        sensitivityMap.getAllFrames(), sensitivityMap.getNFrames(), &p,
                                        &saveSubiteration, &target),
                     "OSEM_ResoReco");
  // FIR's filter leaves the last frame active, the loop the last subset's
  const bool filtered = params.fwhmXYZ[0] > 0.0 && params.fwhmXYZ[1] > 0.0 && params.fwhmXYZ[2] > 0.0;
  if (params.nIterations > 0)
  {
    sensitivityMap.setActiveFrame(params.nSubsets - 1);
  }
  else if (filtered)
  {
    sensitivityMap.setActiveFrame(sensitivityMap.getNFrames() - 1);
  }
}
}  // namespace reconAlgos
