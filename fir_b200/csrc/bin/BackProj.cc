// FIR_BackProj <projection .hs> <scanner file> <volume template .h33> <output name>
// Backprojection of a sinogram into a single-frame volume (FIR:
// src_bin/BackProj.cc).  All four arguments are required.
#include <runtime.h>
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <console.h>
#include <projections.h>

int main(int argc, char** argv)
{
  try
  {
    if (argc < 5)
    {
      error("Requires four input arguments");
    }
    ProjData proj(argv[1], ProjData::ConstructionMode::READ_DATA);
    ScannerData scanner(argv[2]);
    VolData vol(argv[3], VolData::ConstructionMode::ALLOCATE);
    projections::backward(proj, scanner, vol);
    vol.write(argv[4]);
  }
  catch (const std::exception& ex)
  {
    std::cerr << ex.what();
    return EXIT_FAILURE;
  }
  fir_runtime::reportTiming("FIR_BackProj");
  return EXIT_SUCCESS;
}
