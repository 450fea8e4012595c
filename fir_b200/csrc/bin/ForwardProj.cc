// FIR_ForwardProj <parameter file>: forward projection of the frames of a
// volume (FIR: src_bin/ForwardProj.cc).  Parameter file:
//   !FORWARD PROJECTION PARAMETERS :=
//   input volume file := <.h33>            (required)
//   scanner file := <.scan>                (required)
//   output projection header := <.hs>      (required; a template, no data)
//   output projection file name := <name>  (required)
//   frames to project := {0, 2}            (optional; default all frames)
//   mask volume file := <.h33>             (optional; voxels with mask <= 0 are zeroed)
//   !END OF FORWARD PROJECTION PARAMETERS :=
// With several frames (or an explicit frame list) the outputs are
// <name>_frame_<k>.
#include <runtime.h>
#include <KeyParser.h>
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <console.h>
#include <operations.h>
#include <projections.h>
#include <tools.h>

#include <numeric>
#include <optional>

int main(int argc, char** argv)
{
  try
  {
    echo("=== FIR_ForwardProj (B200) ===");
    if (argc < 2)
    {
      error("Parameter file missing");
    }
    std::string volFile, scannerFile, projHeader, projName, maskFile;
    std::vector<int> frames;
    KeyParser kp;
    kp.addStartKey("!FORWARD PROJECTION PARAMETERS");
    kp.addKey("input volume file", &volFile);
    kp.addKey("scanner file", &scannerFile);
    kp.addKey("output projection header", &projHeader);
    kp.addKey("output projection file name", &projName);
    kp.addKey("frames to project", &frames);
    kp.addKey("mask volume file", &maskFile);
    kp.addStopKey("!END OF FORWARD PROJECTION PARAMETERS");
    kp.parse(argv[1]);
    if (volFile.empty())
    {
      error("No input volume file provided");
    }
    if (scannerFile.empty())
    {
      error("No scanner file provided");
    }
    if (projHeader.empty())
    {
      error("No output projection header provided");
    }
    if (projName.empty())
    {
      error("No output projection file name provided");
    }

    VolData vol(volFile, VolData::ConstructionMode::READ_DATA);
    bool single;
    if (frames.empty())
    {
      single = vol.getNFrames() == 1;
      frames.resize(vol.getNFrames());
      std::iota(frames.begin(), frames.end(), 0);
    }
    else
    {
      single = false;
      for (int f : frames)
      {
        if (!(f >= 0 && f < vol.getNFrames()))
        {
          error("Frame indices must be between 0 and ", vol.getNFrames() - 1);
        }
      }
    }
    std::optional<VolData> mask;
    if (!maskFile.empty())
    {
      mask.emplace(maskFile, VolData::ConstructionMode::READ_DATA);
    }
    ScannerData scanner(scannerFile);
    ProjData proj(projHeader, ProjData::ConstructionMode::ALLOCATE);
    for (int f : frames)
    {
      vol.setActiveFrame(f);
      if (mask)
      {
        operations::applyMask(vol, *mask);
      }
      projections::forward(vol, scanner, proj);
      proj.write(single ? projName : projName + "_frame_" + std::to_string(f));
    }
  }
  catch (const std::exception& ex)
  {
    std::cerr << ex.what();
    return EXIT_FAILURE;
  }
  fir_runtime::reportTiming("FIR_ForwardProj");
  return EXIT_SUCCESS;
}
