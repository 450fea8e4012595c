// FIR_OSEM <parameter file> [recompute sensitivity 0|1] [recompute attenuation 0|1]
// OSEM reconstruction (FIR: src_bin/OSEM.cc), same parameter keys and flags:
//   !OSEM PARAMETERS :=
//   input projection file := <.hs>          (required)
//   scanner file := <.scan>                 (required)
//   output volume header := <.h33>          (required; its data, if any, is the start image)
//   output volume file name := <name>       (required)
//   number of iterations := 1
//   number of subsets := 1                  (must divide the number of views)
//   save interval := 0                      (write <name>_subiter_<k> every k sub-iterations)
//   cut radius in mm := 0
//   convolution interval := 0
//   convolution FHWM XYZ in mm := {0, 0, 0} (FIR's spelling of the key)
//   sensitivity map volume := <name>        (read if present, else computed and written)
//   bias projection := <.hs>
//   attenuation volume in HU := <.h33>
//   attenuation correction factors := <name> (read if present, else computed and written)
//   !END OF OSEM PARAMETERS :=
// A flag that does not start with '0' means "recompute" (both default to 1).
#include <runtime.h>
#include <KeyParser.h>
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <console.h>
#include <operations.h>
#include <projections.h>
#include <reconAlgos.h>

#include <fstream>
#include <optional>

namespace
{
bool fileExists(const std::string& f)
{
  std::ifstream s(f);
  return s.good();
}
}  // namespace

int main(int argc, char** argv)
{
  try
  {
    echo("=== FIR_OSEM (B200) ===");
    if (argc < 2)
    {
      error("Parameter file missing");
    }
    std::string projFile, scannerFile, volHeader, volName, sensFile, biasFile, huFile, acfFile;
    OSEMCoreParams prm;
    KeyParser kp;
    kp.addStartKey("!OSEM PARAMETERS");
    kp.addKey("input projection file", &projFile);
    kp.addKey("scanner file", &scannerFile);
    kp.addKey("output volume header", &volHeader);
    kp.addKey("output volume file name", &volName);
    kp.addKey("number of iterations", &prm.nIterations);
    kp.addKey("number of subsets", &prm.nSubsets);
    kp.addKey("save interval", &prm.saveInterval);
    kp.addKey("cut radius in mm", &prm.cutRadius);
    kp.addKey("convolution interval", &prm.convolutionInterval);
    kp.addKey("convolution FHWM XYZ in mm", &prm.fwhmXYZ);
    kp.addKey("sensitivity map volume", &sensFile);
    kp.addKey("bias projection", &biasFile);
    kp.addKey("attenuation volume in HU", &huFile);
    kp.addKey("attenuation correction factors", &acfFile);
    kp.addStopKey("!END OF OSEM PARAMETERS");
    kp.parse(argv[1]);
    if (projFile.empty())
    {
      error("No input projection file provided");
    }
    if (scannerFile.empty())
    {
      error("No scanner file provided");
    }
    if (volHeader.empty())
    {
      error("No output volume header provided");
    }
    if (volName.empty())
    {
      error("No output volume file name provided");
    }

    bool recomputeSens = argc > 2 ? argv[2][0] != '0' : true;
    bool recomputeAcf = argc > 3 ? argv[3][0] != '0' : true;
    if (!recomputeSens)
    {
      // recompute anyway when there is no file to read it from
      recomputeSens = sensFile.empty() || !fileExists(sensFile);
    }
    const bool acfExists = !acfFile.empty() && fileExists(acfFile);

    ProjData proj(projFile, ProjData::ConstructionMode::READ_DATA);
    proj.checkNSubsets(prm.nSubsets);
    ScannerData scanner(scannerFile);
    VolData vol(volHeader, VolData::ConstructionMode::READ_DATA_IF_PROVIDED, 1.0);

    VolData sens;
    if (recomputeSens)
    {
      echo("Computing sensitivity map");
      sens.allocateAsMultiVol(vol, prm.nSubsets);
      projections::computeSensitivityVol(proj, scanner, sens, prm.nSubsets);
      if (!sensFile.empty())
      {
        printQuotedValue("Saving sensitivity map to file", sensFile);
        sens.write(sensFile);
      }
    }
    else
    {
      printQuotedValue("Reading sensitivity map from file", sensFile);
      sens.read(sensFile, VolData::ConstructionMode::READ_DATA);
      if (sens.getHeader() != vol.getHeader())
      {
        error("Sensitivity volume provided doesn't fit with output volume provided");
      }
    }

    std::optional<ProjData> bias;
    if (!biasFile.empty())
    {
      printQuotedValue("Reading bias projection from file", biasFile);
      bias.emplace(biasFile, ProjData::ConstructionMode::READ_DATA);
    }

    // Attenuation correction: the data are multiplied by exp(line integral
    // of mu) (src_bin/OSEM.cc:262-338)
    if (!huFile.empty() || acfExists)
    {
      if (!recomputeAcf && !huFile.empty() && !acfExists)
      {
        recomputeAcf = true;
      }
      if (recomputeAcf && huFile.empty() && acfExists)
      {
        recomputeAcf = false;
      }
      ProjData acf;
      if (recomputeAcf)
      {
        echo("Computing attenuation correction factors");
        VolData mu(huFile, VolData::ConstructionMode::READ_DATA);
        operations::HounsfieldToMuMap(mu);
        operations::cutCircle(mu, prm.cutRadius);
        acf.copy(proj, ProjData::ConstructionMode::INITIALIZE);
        projections::forward(mu, scanner, acf);
        acf.exponential();
        if (!acfFile.empty())
        {
          printQuotedValue("Saving attenuation correction factors to file", acfFile);
          acf.write(acfFile);
        }
      }
      else
      {
        printQuotedValue("Reading attenuation correction factors from file", acfFile);
        acf.read(acfFile, ProjData::ConstructionMode::READ_DATA);
      }
      proj *= acf;
    }

    reconAlgos::OSEM(proj, scanner, vol, volName, prm, sens, bias);
    printQuotedValue("Saving reconstructed volume to file", volName);
    vol.write(volName);
  }
  catch (const std::exception& ex)
  {
    std::cerr << ex.what();
    return EXIT_FAILURE;
  }
  fir_runtime::reportTiming("FIR_OSEM");
  return EXIT_SUCCESS;
}
