// operations:: entry points over the C ABI (FIR: src_lib/operations.cc).
#include <console.h>
#include <operations.h>
#include <runtime.h>

namespace operations
{
void convolve(VolData& vol, std::vector<float> fwhmXYZ, float cutRadius)
{
  if (fwhmXYZ.size() < 3)
  {
    error("convolution FWHM must have three elements");
  }
  if (!(fwhmXYZ[0] > 0.0 && fwhmXYZ[1] > 0.0 && fwhmXYZ[2] > 0.0))
  {
    return;
  }
  const int nFrames = vol.getNFrames();
  const fir_vol_desc vd = fir_runtime::volDesc(vol, nFrames);
  fir_runtime::check(fir_convolve(fir_runtime::context(), &vd, vol.getAllFrames(), fwhmXYZ.data(), cutRadius),
                     "convolution");
  // FIR's frame loop leaves the last frame active (operations.cc:101-103)
  vol.setActiveFrame(nFrames - 1);
}

void cutCircle(VolData& vol, float cutRadius)
{
  if (!(cutRadius > 0.0))
  {
    return;
  }
  const fir_vol_desc vd = fir_runtime::volDesc(vol, 1);
  fir_runtime::check(fir_cut_circle(fir_runtime::context(), &vd, vol.getDataArray(), cutRadius), "cut");
}

void applyMask(VolData& vol, VolData& maskVol)
{
  if (vol.getHeader() != maskVol.getHeader())
  {
    error("Mask volume not the same size");
  }
  const fir_vol_desc vd = fir_runtime::volDesc(vol, 1);
  fir_runtime::check(fir_apply_mask(fir_runtime::context(), &vd, vol.getDataArray(), maskVol.getDataArray()),
                     "mask");
}

void HounsfieldToMuMap(VolData& vol)
{
  const fir_vol_desc vd = fir_runtime::volDesc(vol, 1);
  fir_runtime::check(fir_hu_to_mu(fir_runtime::context(), &vd, vol.getDataArray()), "HU to mu");
}
}  // namespace operations
