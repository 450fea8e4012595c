// Scanner geometry with FIR's public interface (src_lib/ScannerHeader.h,
// src_lib/ScannerData.h:11-53): crystal/module/rSector description read from a
// "!SCANNER PARAMETERS" file, and the crystal XY / slice Z position tables.
// The tables are computed by the C ABI (fir_scanner_tables), the same code
// that feeds the GPU, so host and device see identical doubles.
#pragma once

#include <fir_cuda.h>
#include <types.h>

#include <string>
#include <vector>

class ProjData;
class VolData;

struct ScannerHeader
{
  std::vector<types::SpatialCoord> crystalDimsXYZ;
  std::vector<int> crystalRepeatNumbersYZ;
  std::vector<types::SpatialCoord> interCrystalDistanceYZ;
  std::vector<types::SpatialCoord> moduleDimsXYZ;
  std::vector<int> moduleRepeatNumbersYZ;
  std::vector<types::SpatialCoord> interModuleDistanceYZ;
  std::vector<types::SpatialCoord> rSectorDimsXYZ;
  int rSectorRepeatNumber;
  types::SpatialCoord rSectorInnerRadius;

  void setDefaults();
  // Validates with FIR's messages and replaces zero module / rSector
  // dimensions by the tight fit (ScannerHeader.cc:26-303).
  void check();
};

struct ScannerGeometry
{
  std::vector<types::SpatialCoord> crystalRepeatVectorYZ;
  std::vector<types::SpatialCoord> moduleRepeatVectorYZ;
  types::SpatialCoord rSectorTranslationX;
  int nRings, nCrystalsPerRing, nCrystals;
  int nSlices;
  int crystalOffset;

  void fill(const ScannerHeader& header);
};

class ScannerData
{
public:
  ScannerData();
  ScannerData(const std::string& scannerFile);

  // Throws unless proj has the scanner's rings and crystals per ring
  void checkProjData(const ProjData& proj) const;

  const types::SpatialCoords2D* getCrystalXYPositionVector() const { return mXY.data(); }
  const types::SpatialCoord* getSliceZPositionVector() const { return mZ.data(); }

  void printContent() const;
  void printCrystalPositions() const;
  void printBinInfo(int seg, int view, int axialCoord, int tangCoord, int crystal1, int slice1, int crystal2,
                    int slice2, const VolData& vol, types::PathElement* pathElementsArray = 0,
                    types::VoxelValue line = 0) const;
  void getCrystalCoordinates(int rSectorID, int moduleID, int crystalID, int* ring, int* crystal) const;

  const ScannerHeader& getHeader() const { return mHeader; }
  const ScannerGeometry& getGeometry() const { return mGeometry; }
  // The header as a C-ABI descriptor
  fir_scanner_desc descriptor() const;

private:
  void computeTables();

  ScannerHeader mHeader{};
  ScannerGeometry mGeometry{};
  std::vector<types::SpatialCoords2D> mXY;
  std::vector<types::SpatialCoord> mZ;
};
