// Multi-frame volume with FIR's public interface (src_lib/VolHeader.h,
// src_lib/VolData.h:9-157): float voxels, frames contiguous in one host
// allocation, a mutable active frame, Interfile I/O, and FIR's voxel-wise
// arithmetic with 1e-5 gates.  The projectors and OSEM that consume these
// volumes run on the GPU through the C ABI (include/fir_cuda.h).
#pragma once

#include <types.h>

#include <string>
#include <vector>

struct VolHeader
{
  types::VolSize volSize;
  types::VoxelExtent voxelExtent;
  // x,y: centre of the first voxel; z: offset of the volume centre
  types::SpatialCoords3D volOffset;
  int nFrames;

  bool operator==(const VolHeader& rhs) const
  {
    // the number of frames is not compared (VolHeader.inl:6-12)
    return volSize == rhs.volSize && voxelExtent == rhs.voxelExtent && volOffset == rhs.volOffset;
  }
  bool operator!=(const VolHeader& rhs) const { return !(*this == rhs); }

  void setDefaults();
  void check() const;
};

struct VolGeometry
{
  types::VolExtent volExtent;
  int nVoxelsPerFrame;
  int nVoxelsTotal;

  void fill(const VolHeader& header);
};

class VolData
{
public:
  enum class ConstructionMode
  {
    ALLOCATE,
    INITIALIZE,
    READ_DATA,
    READ_DATA_IF_PROVIDED
  };

  VolData();
  VolData(const std::string& inputVolFile, ConstructionMode mode = ConstructionMode::READ_DATA,
          types::VoxelValue initValue = 0.0);
  VolData(const VolData& vol, ConstructionMode mode = ConstructionMode::READ_DATA,
          types::VoxelValue initValue = 0.0);
  VolData(const VolHeader& header);
  ~VolData() = default;

  VolData& operator=(const VolData&) = delete;
  VolData& operator=(VolData&&) = default;
  VolData(VolData&&) = default;

  void read(const std::string& headerFileName, ConstructionMode mode = ConstructionMode::READ_DATA,
            types::VoxelValue initValue = 0.0);
  void copy(const VolData& vol, ConstructionMode mode = ConstructionMode::READ_DATA,
            types::VoxelValue initValue = 0.0);
  // Writes <name>.h33 (header) and <name>.i33 (FLOAT 4 LITTLEENDIAN), all frames
  void write(const std::string& outputVolFile) const;

  void allocateAsMultiVol(const VolData& templateVol, int nFrames);
  void allocateSingleFrameFromMultiVol(VolData& templateVol);

  void printContent() const;
  void checkNFrames(int nFrames) const;

  void assign(const VolData& vol);
  void assignFrame(const VolData& vol, int frame);
  void setAllVoxels(types::VoxelValue value = 0.0);
  void setAllVoxelsAllFrames(types::VoxelValue value = 0.0);

  // Active-frame arithmetic: x <- x op y if both exceed 1e-5, else 0
  VolData& operator*=(const VolData& inputVol);
  VolData& operator/=(const VolData& inputVol);

  void setActiveFrame(int frame) const;
  int getActiveFrame() const { return mActiveFrame; }

  // Line integral along a path array terminated by coord == -1
  types::VoxelValue computeLineIntegral(types::PathElement* pathElementsArray) const;
  void projectLineIntegral(types::PathElement* pathElementsArray, types::VoxelValue line);

  const VolHeader& getHeader() const { return mHeader; }
  int getNFrames() const { return mHeader.nFrames; }
  const types::VolExtent& getVolExtent() const { return mGeometry.volExtent; }
  int getNVoxelsPerFrame() const { return mGeometry.nVoxelsPerFrame; }
  bool isAllocated() const { return !mData.empty(); }
  // Voxels of the active frame
  types::VoxelValue* getDataArray() const { return mActive; }
  // All frames, contiguous
  types::VoxelValue* getAllFrames() const { return const_cast<types::VoxelValue*>(mData.data()); }

  void setVoxel(int i, int j, int k, types::VoxelValue value)
  {
    mActive[i + j * mHeader.volSize.nPixelsX + k * mHeader.volSize.nPixelsX * mHeader.volSize.nPixelsY] = value;
  }
  types::VoxelValue getVoxel(int i, int j, int k) const
  {
    return mActive[i + j * mHeader.volSize.nPixelsX + k * mHeader.volSize.nPixelsX * mHeader.volSize.nPixelsY];
  }

private:
  void allocate(bool initialize = true, types::VoxelValue initValue = 0.0);

  VolHeader mHeader{};
  VolGeometry mGeometry{};
  mutable int mActiveFrame = 0;
  mutable types::VoxelValue* mActive = nullptr;
  std::vector<types::VoxelValue> mData;
};
