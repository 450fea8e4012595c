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

// FIR's resolution-modelling variant as FIR runs it (reconAlgos.cc:203-367),
// including its order of operations: the sensitivity is filtered once, the
// estimate used in the projection is the unfiltered image, the filtered
// backprojection multiplies the image after the image (not the
// backprojection) is divided by the sensitivity.
void OSEM_ResoReco(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol,
                   const std::string& outputVolFileName, const OSEMCoreParams& params, VolData& sensitivityMap,
                   const std::optional<ProjData>& biasProj)
{
  echo("OSEM_ResoReco:");
  scanner.checkProjData(inputProj);
  inputProj.checkNSubsets(params.nSubsets);
  checkSensitivity(sensitivityMap, outputVol, params.nSubsets);
  const fir_osem_params p = toParams(params);
  const bool convolveFlag = params.convolutionInterval > 0 && params.fwhmXYZ[0] > 0.0 &&
                            params.fwhmXYZ[1] > 0.0 && params.fwhmXYZ[2] > 0.0;
  fir_runtime::useScanner(scanner);
  const fir_vol_desc vd = fir_runtime::volDesc(outputVol, 1);
  const fir_proj_desc pd = fir_runtime::projDesc(inputProj);

  VolData backProj(outputVol, VolData::ConstructionMode::INITIALIZE, 0.0);
  operations::cutCircle(outputVol, params.cutRadius);
  operations::convolve(sensitivityMap, params.fwhmXYZ, params.cutRadius);
  VolData blur(outputVol, VolData::ConstructionMode::READ_DATA);
  const int nSubiterations = params.nIterations * params.nSubsets;
  for (int iter = 0; iter < params.nIterations; ++iter)
  {
    print("Iteration ", iter + 1, " of ", params.nIterations);
    for (int subset = 0; subset < params.nSubsets; ++subset)
    {
      const int subiter = iter * params.nSubsets + subset + 1;
      operations::convolve(blur, params.fwhmXYZ, params.cutRadius);
      fir_runtime::check(fir_ratio_backprojection(fir_runtime::context(), &pd, inputProj.getBins(),
                                                  biasProj ? biasProj->getBins() : nullptr, &vd,
                                                  outputVol.getDataArray(), backProj.getDataArray(),
                                                  params.nSubsets, subset),
                         "ratio backprojection");
      operations::convolve(backProj, params.fwhmXYZ, params.cutRadius);
      sensitivityMap.setActiveFrame(subset);
      outputVol /= sensitivityMap;
      outputVol *= backProj;
      if (convolveFlag && subiter % params.convolutionInterval == 0)
      {
        operations::convolve(outputVol, params.fwhmXYZ, params.cutRadius);
      }
      operations::cutCircle(outputVol, params.cutRadius);
      if (subiter != nSubiterations)
      {
        blur.assign(outputVol);
      }
      if (p.save_interval > 0 && subiter % p.save_interval == 0 && subiter != nSubiterations)
      {
        outputVol.write(outputVolFileName + "_subiter_" + std::to_string(subiter));
      }
    }
  }
}
}  // namespace reconAlgos
