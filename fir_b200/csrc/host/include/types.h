// Data types of FIR's public API (src_lib/types.h:7-76), kept under the same
// names so that code written against FIR compiles unchanged.  Geometry is
// double, voxel and bin values are float, sizes and indices are int.
#pragma once

namespace types
{
using Size = int;
using Index = Size;

using SpatialExtent = double;
using SpatialCoord = SpatialExtent;

using VoxelValue = float;
using BinValue = float;

struct VolSize
{
  Size nPixelsX;
  Size nPixelsY;
  Size nSlices;

  Size nVoxelsTotal() const { return nPixelsX * nPixelsY * nSlices; }
  bool operator==(const VolSize& o) const
  {
    return nPixelsX == o.nPixelsX && nPixelsY == o.nPixelsY && nSlices == o.nSlices;
  }
};

struct VoxelExtent
{
  SpatialExtent pixelWidth;
  SpatialExtent pixelHeight;
  SpatialExtent sliceThickness;

  bool operator==(const VoxelExtent& o) const
  {
    return pixelWidth == o.pixelWidth && pixelHeight == o.pixelHeight && sliceThickness == o.sliceThickness;
  }
};

struct VolExtent
{
  SpatialExtent sliceWidth;
  SpatialExtent sliceHeight;
  SpatialExtent volDepth;
};

inline VolExtent operator*(const VolSize& s, const VoxelExtent& e)
{
  return {s.nPixelsX * e.pixelWidth, s.nPixelsY * e.pixelHeight, s.nSlices * e.sliceThickness};
}

struct SpatialCoords3D
{
  SpatialCoord x;
  SpatialCoord y;
  SpatialCoord z;

  bool operator==(const SpatialCoords3D& o) const { return x == o.x && y == o.y && z == o.z; }
};

struct SpatialCoords2D
{
  SpatialCoord x;
  SpatialCoord y;
};

struct PathElement
{
  Index coord;
  SpatialExtent length;
};
}  // namespace types
