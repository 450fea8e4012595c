// Sinogram data model with FIR's public interface (src_lib/ProjHeader.h,
// src_lib/ProjData.h:23-170).  Bins are float, stored as one contiguous
// block in file order (segments -segOffset..+segOffset, each
// [view][axial][tang]); getDataArray() gives FIR's per-segment pointers into
// that block.  Header validation and derived geometry come from the C ABI
// (fir_proj_geometry), so both sides of the boundary agree.
#pragma once

#include <types.h>

#include <string>
#include <tuple>
#include <vector>

struct ProjHeader
{
  int nRings;
  int nCrystalsPerRing;
  int segmentSpan;
  int nSegments;
  int nTangCoords;

  bool operator==(const ProjHeader& rhs) const
  {
    return nRings == rhs.nRings && nCrystalsPerRing == rhs.nCrystalsPerRing && segmentSpan == rhs.segmentSpan &&
           nSegments == rhs.nSegments && nTangCoords == rhs.nTangCoords;
  }

  void setDefaults();
  // Throws FIR's messages; replaces nTangCoords = 0 by its maximum.
  void check();
};

struct ProjGeometry
{
  int nBins;
  int segOffset;
  int tangCoordOffset;
  std::vector<int> nAxialCoords;
  int nViews;
  int halfSegmentSpan;
  int maxRingDiff;

  int getNAxialCoords(int seg) const { return nAxialCoords[seg + segOffset]; }
  void fill(const ProjHeader& header);
};

class ProjData
{
public:
  enum class ConstructionMode
  {
    ALLOCATE,
    INITIALIZE,
    READ_DATA
  };

  ProjData();
  ProjData(const std::string& inputProjFile, ConstructionMode mode = ConstructionMode::READ_DATA,
           types::BinValue initValue = 0.0);
  ProjData(const ProjData& proj, ConstructionMode mode = ConstructionMode::READ_DATA,
           types::BinValue initValue = 0.0);
  ~ProjData() = default;
  ProjData& operator=(ProjData&&) = default;
  ProjData(ProjData&&) = default;

  void read(const std::string& headerFileName, ConstructionMode mode = ConstructionMode::READ_DATA,
            types::BinValue initValue = 0.0);
  void copy(const ProjData& proj, ConstructionMode mode = ConstructionMode::READ_DATA,
            types::BinValue initValue = 0.0);
  // Writes <name>.hs and <name>.s
  void write(const std::string& outputProjFile) const;
  void printContent() const;

  void checkNSubsets(int nSubsets) const;
  void setAllBins(types::BinValue value = 0.0);

  // Bin coordinates -> slice indices / crystal indices (ProjData.cc:198-340)
  std::tuple<int, int> getCrystalAxialCoord(int seg, int axialCoord) const;
  std::tuple<int, int> getCrystalAngCoord(int view, int tangCoord) const;

  // Crystal pair -> bin coordinates (ProjData.cc:342-479); false when the LOR
  // lies outside the allocated segments or tangential range.
  bool getBinCoordinates(int crystalAxialCoord1, int crystalAngCoord1, int crystalAxialCoord2, int crystalAngCoord2,
                         int* seg, int* view, int* axialCoord, int* tangCoord) const;

  // Bin-wise arithmetic on the GPU: product with 1e-5 gates, exponential,
  // and the span > 1 weights of ProjData.cc:541-615
  ProjData& operator*=(const ProjData& inputProj);
  void exponential();
  void rebinWeight();

  const ProjHeader& getHeader() const { return mHeader; }
  const ProjGeometry& getGeometry() const { return mGeometry; }
  types::BinValue** getDataArray() const { return const_cast<types::BinValue**>(mSegments.data()); }
  // All bins in file order
  types::BinValue* getBins() const { return const_cast<types::BinValue*>(mData.data()); }

  void setBin(int seg, int view, int axialCoord, int tangCoord, types::BinValue value)
  {
    at(seg, view, axialCoord, tangCoord) = value;
  }
  types::BinValue getBin(int seg, int view, int axialCoord, int tangCoord) const
  {
    return const_cast<ProjData*>(this)->at(seg, view, axialCoord, tangCoord);
  }
  void incrementBin(int seg, int view, int axialCoord, int tangCoord) { at(seg, view, axialCoord, tangCoord)++; }
  void weightBin(int seg, int view, int axialCoord, int tangCoord, types::BinValue weight)
  {
    at(seg, view, axialCoord, tangCoord) *= weight;
  }

private:
  types::BinValue& at(int seg, int view, int axialCoord, int tangCoord)
  {
    const int nax = mGeometry.getNAxialCoords(seg);
    return mSegments[seg + mGeometry.segOffset][view * nax * mHeader.nTangCoords + axialCoord * mHeader.nTangCoords +
                                                tangCoord + mGeometry.tangCoordOffset];
  }
  void allocate(bool initialize, types::BinValue initValue);

  ProjHeader mHeader{};
  ProjGeometry mGeometry{};
  std::vector<types::BinValue> mData;
  std::vector<types::BinValue*> mSegments;
};
