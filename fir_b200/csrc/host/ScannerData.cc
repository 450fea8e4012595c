// Scanner header parsing, validation and position tables (FIR's
// ScannerHeader.cc, ScannerInterfileReader.cc, ScannerData.cc); validation and
// tables are delegated to the C ABI so the host and the GPU agree exactly.
#include <KeyParser.h>
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <console.h>
#include <macros.h>

#include <cstdio>

void ScannerHeader::setDefaults()
{
  crystalDimsXYZ.assign(3, 0.0);
  crystalRepeatNumbersYZ.assign(2, 1);
  interCrystalDistanceYZ.assign(2, 0.0);
  moduleDimsXYZ.assign(3, 0.0);
  moduleRepeatNumbersYZ.assign(2, 1);
  interModuleDistanceYZ.assign(2, 0.0);
  rSectorDimsXYZ.assign(3, 0.0);
  rSectorRepeatNumber = 0;
  rSectorInnerRadius = 0.0;
}

namespace
{
void needSize(const char* key, size_t have, size_t want)
{
  if (have != want)
  {
    error("\"", key, "\" must contain ", want == 3 ? "three" : "two", " elements");
  }
}
}  // namespace

void ScannerHeader::check()
{
  needSize("crystal dimensions XYZ in mm", crystalDimsXYZ.size(), 3);
  needSize("crystal repeat numbers YZ", crystalRepeatNumbersYZ.size(), 2);
  needSize("inter-crystal distance YZ in mm", interCrystalDistanceYZ.size(), 2);
  needSize("module dimensions XYZ in mm", moduleDimsXYZ.size(), 3);
  needSize("module repeat numbers YZ", moduleRepeatNumbersYZ.size(), 2);
  needSize("inter-module distance YZ in mm", interModuleDistanceYZ.size(), 2);
  needSize("rSector dimensions XYZ in mm", rSectorDimsXYZ.size(), 3);
  fir_scanner_desc d;
  for (int i = 0; i < 3; ++i)
  {
    d.crystal_dims[i] = crystalDimsXYZ[i];
    d.module_dims[i] = moduleDimsXYZ[i];
    d.rsector_dims[i] = rSectorDimsXYZ[i];
  }
  for (int i = 0; i < 2; ++i)
  {
    d.crystal_repeat[i] = crystalRepeatNumbersYZ[i];
    d.inter_crystal[i] = interCrystalDistanceYZ[i];
    d.module_repeat[i] = moduleRepeatNumbersYZ[i];
    d.inter_module[i] = interModuleDistanceYZ[i];
  }
  d.rsector_repeat = rSectorRepeatNumber;
  d.rsector_inner_radius = rSectorInnerRadius;
  if (fir_scanner_tables(&d, nullptr, nullptr, nullptr, nullptr) != FIR_OK)
  {
    error(fir_last_error());
  }
  // tight-fit defaults (ScannerHeader.cc:213-303)
  const double minMod[3] = {
    crystalDimsXYZ[0],
    crystalDimsXYZ[1] * crystalRepeatNumbersYZ[0] + interCrystalDistanceYZ[0] * (crystalRepeatNumbersYZ[0] - 1),
    crystalDimsXYZ[2] * crystalRepeatNumbersYZ[1] + interCrystalDistanceYZ[1] * (crystalRepeatNumbersYZ[1] - 1)};
  for (int i = 0; i < 3; ++i)
  {
    if (moduleDimsXYZ[i] == 0.0)
    {
      moduleDimsXYZ[i] = minMod[i];
    }
  }
  const double minRs[3] = {
    moduleDimsXYZ[0],
    moduleDimsXYZ[1] * moduleRepeatNumbersYZ[0] + interModuleDistanceYZ[0] * (moduleRepeatNumbersYZ[0] - 1),
    moduleDimsXYZ[2] * moduleRepeatNumbersYZ[1] + interModuleDistanceYZ[1] * (moduleRepeatNumbersYZ[1] - 1)};
  for (int i = 0; i < 3; ++i)
  {
    if (rSectorDimsXYZ[i] == 0.0)
    {
      rSectorDimsXYZ[i] = minRs[i];
    }
  }
}

void ScannerGeometry::fill(const ScannerHeader& h)
{
  crystalRepeatVectorYZ = {h.crystalDimsXYZ[1] + h.interCrystalDistanceYZ[0],
                           h.crystalDimsXYZ[2] + h.interCrystalDistanceYZ[1]};
  moduleRepeatVectorYZ = {h.moduleDimsXYZ[1] + h.interModuleDistanceYZ[0],
                          h.moduleDimsXYZ[2] + h.interModuleDistanceYZ[1]};
  rSectorTranslationX = h.rSectorInnerRadius + h.rSectorDimsXYZ[0] / 2;
  nCrystalsPerRing = h.crystalRepeatNumbersYZ[0] * h.moduleRepeatNumbersYZ[0] * h.rSectorRepeatNumber;
  nRings = h.crystalRepeatNumbersYZ[1] * h.moduleRepeatNumbersYZ[1];
  nCrystals = nRings * nCrystalsPerRing;
  nSlices = 2 * nRings - 1;
  crystalOffset = h.moduleRepeatNumbersYZ[0] * h.crystalRepeatNumbersYZ[0] / 2;
}

ScannerData::ScannerData() { mHeader.setDefaults(); }

ScannerData::ScannerData(const std::string& scannerFile) : ScannerData()
{
  KeyParser kp;
  kp.addStartKey("!SCANNER PARAMETERS");
  kp.addKey("crystal dimensions XYZ in mm", &mHeader.crystalDimsXYZ);
  kp.addKey("crystal repeat numbers YZ", &mHeader.crystalRepeatNumbersYZ);
  kp.addKey("inter-crystal distance YZ in mm", &mHeader.interCrystalDistanceYZ);
  kp.addKey("module dimensions XYZ in mm", &mHeader.moduleDimsXYZ);
  kp.addKey("module repeat numbers YZ", &mHeader.moduleRepeatNumbersYZ);
  kp.addKey("inter-module distance YZ in mm", &mHeader.interModuleDistanceYZ);
  kp.addKey("rSector dimensions XYZ in mm", &mHeader.rSectorDimsXYZ);
  kp.addKey("rSector repeat number", &mHeader.rSectorRepeatNumber);
  kp.addKey("rSector inner radius in mm", &mHeader.rSectorInnerRadius);
  kp.addStopKey("!END OF SCANNER PARAMETERS");
  kp.parse(scannerFile);
  mHeader.check();
  mGeometry.fill(mHeader);
  computeTables();
}

fir_scanner_desc ScannerData::descriptor() const
{
  fir_scanner_desc d;
  for (int i = 0; i < 3; ++i)
  {
    d.crystal_dims[i] = mHeader.crystalDimsXYZ[i];
    d.module_dims[i] = mHeader.moduleDimsXYZ[i];
    d.rsector_dims[i] = mHeader.rSectorDimsXYZ[i];
  }
  for (int i = 0; i < 2; ++i)
  {
    d.crystal_repeat[i] = mHeader.crystalRepeatNumbersYZ[i];
    d.inter_crystal[i] = mHeader.interCrystalDistanceYZ[i];
    d.module_repeat[i] = mHeader.moduleRepeatNumbersYZ[i];
    d.inter_module[i] = mHeader.interModuleDistanceYZ[i];
  }
  d.rsector_repeat = mHeader.rSectorRepeatNumber;
  d.rsector_inner_radius = mHeader.rSectorInnerRadius;
  return d;
}

void ScannerData::computeTables()
{
  const fir_scanner_desc d = descriptor();
  std::vector<double> xy(2 * static_cast<size_t>(mGeometry.nCrystalsPerRing));
  mZ.assign(static_cast<size_t>(mGeometry.nSlices), 0.0);
  if (fir_scanner_tables(&d, xy.data(), mZ.data(), nullptr, nullptr) != FIR_OK)
  {
    error(fir_last_error());
  }
  mXY.resize(static_cast<size_t>(mGeometry.nCrystalsPerRing));
  for (size_t i = 0; i < mXY.size(); ++i)
  {
    mXY[i] = {xy[2 * i], xy[2 * i + 1]};
  }
}

void ScannerData::checkProjData(const ProjData& proj) const
{
  const auto& h = proj.getHeader();
  if (h.nRings != mGeometry.nRings || h.nCrystalsPerRing != mGeometry.nCrystalsPerRing)
  {
    error("Projection must have the same number of rings (", mGeometry.nRings,
          ") and the same number of crystals per ring (", mGeometry.nCrystalsPerRing, ") as the scanner");
  }
}

void ScannerData::printContent() const
{
  echo("= Scanner header:");
  printEmptyLine();
  printVector("crystal dimensions XYZ in mm", mHeader.crystalDimsXYZ);
  printVector("crystal repeat numbers YZ", mHeader.crystalRepeatNumbersYZ);
  printVector("inter-crystal distance YZ in mm", mHeader.interCrystalDistanceYZ);
  printVector("module dimensions XYZ in mm", mHeader.moduleDimsXYZ);
  printVector("module repeat numbers YZ", mHeader.moduleRepeatNumbersYZ);
  printVector("inter-module distance YZ in mm", mHeader.interModuleDistanceYZ);
  printVector("rSector dimensions XYZ in mm", mHeader.rSectorDimsXYZ);
  printValue("rSector repeat number", mHeader.rSectorRepeatNumber);
  printValue("rSector inner radius in mm", mHeader.rSectorInnerRadius);
  printValue("number of rings", mGeometry.nRings);
  printValue("number of crystals per ring", mGeometry.nCrystalsPerRing);
  printValue("number of crystals", mGeometry.nCrystals);
  printValue("number of slices", mGeometry.nSlices);
  printValue("crystal offset", mGeometry.crystalOffset);
  printEmptyLine();
}

void ScannerData::printCrystalPositions() const
{
  echo("Crystal positions in single ring (X , Y):");
  for (const auto& p : mXY)
  {
    std::printf("%.5f , %.5f\n", p.x, p.y);
  }
  printEmptyLine();
  echo("Slice positions in Z:");
  for (double z : mZ)
  {
    std::printf("%.5f\n", z);
  }
  printEmptyLine();
}

void ScannerData::printBinInfo(int seg, int view, int axialCoord, int tangCoord, int crystal1, int slice1,
                               int crystal2, int slice2, const VolData& vol, types::PathElement* path,
                               types::VoxelValue line) const
{
  printValue("seg", seg);
  printValue("view", view);
  printValue("axialCoord", axialCoord);
  printValue("tangCoord", tangCoord);
  printValue("crystal1", crystal1);
  printValue("slice1", slice1);
  printValue("crystal2", crystal2);
  printValue("slice2", slice2);
  std::cout << "X: (" << mXY[crystal1].x << "," << mXY[crystal2].x << ")\n";
  std::cout << "Y: (" << mXY[crystal1].y << "," << mXY[crystal2].y << ")\n";
  std::cout << "Z: (" << mZ[slice1] << "," << mZ[slice2] << ")\n";
  if (path)
  {
    for (int k = 0; path[k].coord != -1; ++k)
    {
      std::cout << (k ? "," : "{") << path[k].coord;
    }
    std::cout << "}\n";
    for (int k = 0; path[k].coord != -1; ++k)
    {
      std::cout << (k ? "," : "{") << path[k].length;
    }
    std::cout << "}\n";
    for (int k = 0; path[k].coord != -1; ++k)
    {
      std::cout << (k ? "," : "{") << vol.getDataArray()[path[k].coord];
    }
    std::cout << "}\n";
  }
  printValue("line", line);
  printEmptyLine();
}

void ScannerData::getCrystalCoordinates(int rSectorID, int moduleID, int crystalID, int* ring, int* crystal) const
{
  const int my = mHeader.moduleRepeatNumbersYZ[0];
  const int cy = mHeader.crystalRepeatNumbersYZ[0];
  const int cz = mHeader.crystalRepeatNumbersYZ[1];
  *ring = (moduleID / my) * cz + crystalID / cy;
  int c = rSectorID * my * cy + (moduleID % my) * cy + (crystalID % cy) - mGeometry.crystalOffset;
  if (c >= mGeometry.nCrystalsPerRing)
  {
    c -= mGeometry.nCrystalsPerRing;
  }
  *crystal = c;
}
