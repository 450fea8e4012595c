// FIR's projector entry points (src_lib/projections.h:9-24), same
// signatures; they run on the GPU through the C ABI (fir_forward,
// fir_backward, fir_sensitivity).
#pragma once

#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>

namespace projections
{
// outputProj <- projection of the active frame of inputVol
void forward(const VolData& inputVol, const ScannerData& scanner, ProjData& outputProj);

// outputVol (nSubsets frames) <- backprojection of each subset's bins
void backward(const ProjData& inputProj, const ScannerData& scanner, VolData& outputVol, int nSubsets = 1);

// initializedSensVol (nSubsets frames) <- backprojection of ones
void computeSensitivityVol(const ProjData& proj, const ScannerData& scanner, VolData& initializedSensVol,
                           int nSubsets = 1);
}  // namespace projections
