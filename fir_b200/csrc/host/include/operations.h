// FIR's image operations (src_lib/operations.h:7-22), same signatures; they
// run on the GPU through the C ABI.
#pragma once

#include <VolData.h>

#include <vector>

namespace operations
{
// Separable Gaussian filter of every frame (FWHM in mm); voxels at radius
// >= cutRadius - 5 * FWHM keep their value when cutRadius > 0.
void convolve(VolData& vol, std::vector<float> fwhmXYZ, float cutRadius);

// Zero the active frame outside radius cutRadius (0: no cut)
void cutCircle(VolData& vol, float cutRadius = 0.0);

// Zero the voxels of the active frame where maskVol <= 0
void applyMask(VolData& vol, VolData& maskVol);

// Hounsfield units to attenuation coefficients in 1/mm (water 0.0096)
void HounsfieldToMuMap(VolData& vol);
}  // namespace operations
