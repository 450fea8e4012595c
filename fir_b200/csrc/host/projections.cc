// projections:: entry points over the C ABI (FIR: src_lib/projections.cc).
#include <console.h>
#include <projections.h>
#include <runtime.h>

namespace projections
{
void forward(const VolData& inputVol, const ScannerData& scanner, ProjData& outputProj)
{
  scanner.checkProjData(outputProj);
  fir_runtime::useScanner(scanner);
  const fir_vol_desc vd = fir_runtime::volDesc(inputVol, 1);
  const fir_proj_desc pd = fir_runtime::projDesc(outputProj);
  fir_runtime::check(fir_forward(fir_runtime::context(), &vd, inputVol.getDataArray(), &pd, outputProj.getBins()),
                     "forward projection");
}

void backward(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol, int nSubsets)
{
  scanner.checkProjData(inputProj);
  inputProj.checkNSubsets(nSubsets);
  outputVol.checkNFrames(nSubsets);
  echo("Back-projection");
  fir_runtime::useScanner(scanner);
  const fir_vol_desc vd = fir_runtime::volDesc(outputVol, nSubsets);
  const fir_proj_desc pd = fir_runtime::projDesc(inputProj);
  fir_runtime::check(fir_backward(fir_runtime::context(), &pd, inputProj.getBins(), &vd, outputVol.getAllFrames(),
                                  nSubsets),
                     "backprojection");
  // FIR leaves the last subset's frame active (projections.cc:134)
  outputVol.setActiveFrame(nSubsets - 1);
}

void computeSensitivityVol(const ProjData& proj, const ScannerData& scanner, VolData& sens, int nSubsets)
{
  scanner.checkProjData(proj);
  proj.checkNSubsets(nSubsets);
  sens.checkNFrames(nSubsets);
  echo("Back-projection");
  fir_runtime::useScanner(scanner);
  const fir_vol_desc vd = fir_runtime::volDesc(sens, nSubsets);
  const fir_proj_desc pd = fir_runtime::projDesc(proj);
  fir_runtime::check(fir_sensitivity(fir_runtime::context(), &pd, &vd, sens.getAllFrames(), nSubsets),
                     "sensitivity");
  sens.setActiveFrame(nSubsets - 1);
}
}  // namespace projections
