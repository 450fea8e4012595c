// Volume data model and its Interfile I/O (.h33 header + raw data), with
// the behaviour of FIR's VolHeader/VolData/VolInterfileReader
// (src_lib/VolHeader.cc, VolData.cc, VolInterfileReader.cc): every number
// format FIR reads (unsigned/signed integers of 1, 2, 4, 8 bytes, floats of
// 4 or 8 bytes, either byte order, data offset), FLOAT 4 LITTLEENDIAN on
// write, and FIR's header keys and "%.7f" doubles.
#include <KeyParser.h>
#include <VolData.h>
#include <console.h>
#include <macros.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>

void VolHeader::setDefaults()
{
  volSize = {0, 0, 0};
  voxelExtent = {0.0, 0.0, 0.0};
  volOffset = {0.0, 0.0, 0.0};
  nFrames = 1;
}

void VolHeader::check() const
{
  if (volSize.nPixelsX <= 0 || volSize.nPixelsY <= 0 || volSize.nSlices <= 0)
  {
    error("Number of voxels must be greater than zero in each dimension");
  }
  if (voxelExtent.pixelWidth <= 0 || voxelExtent.pixelHeight <= 0 || voxelExtent.sliceThickness <= 0)
  {
    error("Voxel extent must be greater than zero in each dimension");
  }
  if (nFrames <= 0)
  {
    error("Number of frames must be greater than zero");
  }
}

void VolGeometry::fill(const VolHeader& h)
{
  volExtent = h.volSize * h.voxelExtent;
  nVoxelsPerFrame = h.volSize.nPixelsX * h.volSize.nPixelsY * h.volSize.nSlices;
  nVoxelsTotal = nVoxelsPerFrame * h.nFrames;
}

namespace
{
bool littleEndianHost()
{
  const int one = 1;
  return *reinterpret_cast<const char*>(&one) == 1;
}

template<typename T>
T byteSwap(T v)
{
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  std::reverse(b, b + sizeof(T));
  std::memcpy(&v, b, sizeof(T));
  return v;
}

std::string upper(std::string s)
{
  for (auto& c : s)
  {
    c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  }
  return s;
}

void prependHeaderDir(const std::string& header, std::string& data)
{
  if (!data.empty() && data[0] != '/')
  {
    const auto slash = header.find_last_of('/');
    if (slash != std::string::npos)
    {
      data.insert(0, header, 0, slash + 1);
    }
  }
}

struct DataParams
{
  std::string file;
  int offset = 0;
  std::string format;
  int bytes = 0;
  std::string order;
};

template<typename T>
void readFrames(const DataParams& p, const VolGeometry& g, int nFrames, float* out, bool swap)
{
  std::ifstream in(p.file, std::ios::binary);
  if (!in.is_open())
  {
    error("Couldn't open file ", p.file);
  }
  in.seekg(p.offset, std::ios::beg);
  std::vector<T> buf(g.nVoxelsPerFrame);
  for (int f = 0; f < nFrames; ++f)
  {
    in.read(reinterpret_cast<char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(T)));
    if (!in)
    {
      error("The number of pixels that were read from the data file (", in.gcount(),
            ") is inferior to the number expected from the header file (", g.nVoxelsTotal, ")");
    }
    float* dst = out + static_cast<size_t>(f) * g.nVoxelsPerFrame;
    for (int i = 0; i < g.nVoxelsPerFrame; ++i)
    {
      dst[i] = static_cast<float>(swap ? byteSwap(buf[i]) : buf[i]);
    }
  }
}

void writeDouble(std::ofstream& os, const char* key, double v)
{
  char s[64];
  std::snprintf(s, sizeof(s), "%.7f", v);
  os << key << " := " << s << "\n";
}

template<typename T>
void writeKey(std::ofstream& os, const char* key, const T& v)
{
  os << key << " := " << v << "\n";
}
}  // namespace

VolData::VolData() { mHeader.setDefaults(); }

VolData::VolData(const std::string& file, ConstructionMode mode, types::VoxelValue init) : VolData()
{
  read(file, mode, init);
}

VolData::VolData(const VolData& vol, ConstructionMode mode, types::VoxelValue init) : VolData()
{
  copy(vol, mode, init);
}

VolData::VolData(const VolHeader& header) : VolData()
{
  header.check();
  mHeader = header;
  mGeometry.fill(mHeader);
  allocate();
}

void VolData::allocate(bool initialize, types::VoxelValue initValue)
{
  mData.assign(static_cast<size_t>(mGeometry.nVoxelsTotal), initialize ? initValue : 0.0f);
  mActiveFrame = 0;
  mActive = mData.data();
}

void VolData::read(const std::string& headerFile, ConstructionMode mode, types::VoxelValue initValue)
{
  DataParams p;
  VolHeader h;
  h.setDefaults();
  KeyParser kp;
  kp.addStartKey("!INTERFILE");
  kp.addKey("name of data file", &p.file);
  kp.addKey("data offset in bytes", &p.offset);
  kp.addKey("number format", &p.format);
  kp.addKey("number of bytes per pixel", &p.bytes);
  kp.addKey("imagedata byte order", &p.order);
  kp.addKey("matrix size [1]", &h.volSize.nPixelsX);
  kp.addKey("matrix size [2]", &h.volSize.nPixelsY);
  kp.addKey("number of slices", &h.volSize.nSlices);
  kp.addKey("scaling factor (mm/pixel) [1]", &h.voxelExtent.pixelWidth);
  kp.addKey("scaling factor (mm/pixel) [2]", &h.voxelExtent.pixelHeight);
  kp.addKey("slice thickness (pixels)", &h.voxelExtent.sliceThickness);
  kp.addKey("first pixel offset (mm) [1]", &h.volOffset.x);
  kp.addKey("first pixel offset (mm) [2]", &h.volOffset.y);
  kp.addKey("first pixel offset (mm) [3]", &h.volOffset.z);
  kp.addKey("number of time frames", &h.nFrames);
  kp.addStopKey("!END OF INTERFILE");
  kp.parse(headerFile);
  prependHeaderDir(headerFile, p.file);

  // VolInterfileReaderParams::check (VolInterfileReader.cc:26-135)
  if (p.offset < 0)
  {
    error("Data offset must not be negative");
  }
  const auto fmt = upper(p.format);
  auto order = upper(p.order);
  int fallback = 0;
  char kind = 0;
  if (fmt == "SHORT FLOAT")
  {
    kind = 'f';
    fallback = p.bytes != 4 ? 4 : 0;
  }
  else if (fmt == "LONG FLOAT")
  {
    kind = 'f';
    fallback = p.bytes != 8 ? 8 : 0;
  }
  else if (fmt == "FLOAT")
  {
    kind = 'f';
    fallback = (p.bytes == 4 || p.bytes == 8) ? 0 : 4;
  }
  else if (fmt == "UNSIGNED INTEGER" || fmt == "SIGNED INTEGER")
  {
    kind = fmt[0] == 'U' ? 'u' : 'i';
    fallback = (p.bytes == 1 || p.bytes == 2 || p.bytes == 4 || p.bytes == 8) ? 0 : 4;
  }
  else
  {
    error("Unrecognized data type name ", fmt);
  }
  if (fallback)
  {
    p.bytes = fallback;
    warning("Invalid value for bytes per pixel. Using default for datatype ", fmt, ", which is ", p.bytes, ".");
  }
  if (order.empty())
  {
    order = littleEndianHost() ? "LITTLEENDIAN" : "BIGENDIAN";
    warning("Invalid value for imagedata byte order. Using default for current machine (LITTLEENDIAN).");
  }
  else if (order != "LITTLEENDIAN" && order != "BIGENDIAN")
  {
    error("Unrecognized byte order", order);
  }
  h.check();
  mHeader = h;
  mGeometry.fill(mHeader);
  allocate(mode == ConstructionMode::INITIALIZE ||
             (mode == ConstructionMode::READ_DATA_IF_PROVIDED && p.file.empty()),
           initValue);
  const bool readIt = mode == ConstructionMode::READ_DATA ||
                      (mode == ConstructionMode::READ_DATA_IF_PROVIDED && !p.file.empty());
  if (!readIt)
  {
    return;
  }
  const bool swap = littleEndianHost() ? order != "LITTLEENDIAN" : order != "BIGENDIAN";
  float* out = mData.data();
  switch (kind)
  {
  case 'f':
    if (p.bytes == 4)
      readFrames<float>(p, mGeometry, mHeader.nFrames, out, swap);
    else
      readFrames<double>(p, mGeometry, mHeader.nFrames, out, swap);
    break;
  case 'u':
    if (p.bytes == 1)
      readFrames<std::uint8_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else if (p.bytes == 2)
      readFrames<std::uint16_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else if (p.bytes == 4)
      readFrames<std::uint32_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else
      readFrames<std::uint64_t>(p, mGeometry, mHeader.nFrames, out, swap);
    break;
  default:
    if (p.bytes == 1)
      readFrames<std::int8_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else if (p.bytes == 2)
      readFrames<std::int16_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else if (p.bytes == 4)
      readFrames<std::int32_t>(p, mGeometry, mHeader.nFrames, out, swap);
    else
      readFrames<std::int64_t>(p, mGeometry, mHeader.nFrames, out, swap);
    break;
  }
}

void VolData::copy(const VolData& vol, ConstructionMode mode, types::VoxelValue initValue)
{
  mHeader = vol.mHeader;
  mGeometry = vol.mGeometry;
  switch (mode)
  {
  case ConstructionMode::ALLOCATE: allocate(false); break;
  case ConstructionMode::INITIALIZE: allocate(true, initValue); break;
  case ConstructionMode::READ_DATA:
    if (!vol.isAllocated())
    {
      error("Mode is READ_DATA and volume to copy isn't allocated");
    }
    mData = vol.mData;
    mActiveFrame = 0;
    mActive = mData.data();
    break;
  case ConstructionMode::READ_DATA_IF_PROVIDED:
    if (vol.isAllocated())
    {
      mData = vol.mData;
      mActiveFrame = 0;
      mActive = mData.data();
    }
    else
    {
      allocate(true, initValue);
    }
    break;
  }
}

void VolData::write(const std::string& outputVolFile) const
{
  if (!isAllocated())
  {
    error("Volume data is not allocated");
  }
  std::filesystem::path hdr(outputVolFile), dat(outputVolFile);
  hdr.replace_extension(".h33");
  dat.replace_extension(".i33");
  std::ofstream os(hdr);
  if (!os.is_open())
  {
    error("Couldn't create file ", hdr.string());
  }
  // Header layout of VolInterfileReader.cc:551-626
  os << "!INTERFILE :=\n\n";
  writeKey(os, "name of data file", dat.filename().string());
  writeKey(os, "data offset in bytes", 0);
  writeKey(os, "number format", "FLOAT");
  writeKey(os, "number of bytes per pixel", 4);
  writeKey(os, "imagedata byte order", "LITTLEENDIAN");
  os << "\n";
  writeKey(os, "number of dimensions", 3);
  os << "\n";
  writeKey(os, "matrix size [1]", mHeader.volSize.nPixelsX);
  writeKey(os, "matrix size [2]", mHeader.volSize.nPixelsY);
  writeKey(os, "matrix size [3]", mHeader.volSize.nSlices);
  writeKey(os, "number of slices", mHeader.volSize.nSlices);
  os << "\n";
  writeDouble(os, "scaling factor (mm/pixel) [1]", mHeader.voxelExtent.pixelWidth);
  writeDouble(os, "scaling factor (mm/pixel) [2]", mHeader.voxelExtent.pixelHeight);
  writeDouble(os, "scaling factor (mm/pixel) [3]", mHeader.voxelExtent.sliceThickness);
  writeDouble(os, "slice thickness (pixels)", mHeader.voxelExtent.sliceThickness);
  os << "\n";
  writeDouble(os, "first pixel offset (mm) [1]", mHeader.volOffset.x);
  writeDouble(os, "first pixel offset (mm) [2]", mHeader.volOffset.y);
  writeDouble(os, "first pixel offset (mm) [3]", mHeader.volOffset.z);
  os << "\n";
  writeKey(os, "number of time frames", mHeader.nFrames);
  os << "\n";
  os << "!END OF INTERFILE :=\n";
  std::ofstream ds(dat, std::ios::binary);
  if (!ds.is_open())
  {
    error("Couldn't create file ", dat.string());
  }
  if (littleEndianHost())
  {
    ds.write(reinterpret_cast<const char*>(mData.data()), static_cast<std::streamsize>(mData.size() * sizeof(float)));
  }
  else
  {
    for (float v : mData)
    {
      const float s = byteSwap(v);
      ds.write(reinterpret_cast<const char*>(&s), sizeof(float));
    }
  }
}

void VolData::allocateAsMultiVol(const VolData& t, int nFrames)
{
  if (nFrames <= 0)
  {
    error("Number of frames must be greater than zero");
  }
  mHeader = t.mHeader;
  mGeometry = t.mGeometry;
  mHeader.nFrames = nFrames;
  mGeometry.nVoxelsTotal = mGeometry.nVoxelsPerFrame * nFrames;
  allocate();
}

void VolData::allocateSingleFrameFromMultiVol(VolData& t)
{
  mHeader = t.mHeader;
  mGeometry = t.mGeometry;
  mHeader.nFrames = 1;
  mGeometry.nVoxelsTotal = mGeometry.nVoxelsPerFrame;
  allocate();
}

void VolData::printContent() const
{
  echo("= Volume header:");
  printEmptyLine();
  printVector<types::Size>("volume size in voxels",
                           {mHeader.volSize.nPixelsX, mHeader.volSize.nPixelsY, mHeader.volSize.nSlices});
  printVector<double>("voxel extent in mm", {mHeader.voxelExtent.pixelWidth, mHeader.voxelExtent.pixelHeight,
                                             mHeader.voxelExtent.sliceThickness});
  printVector<double>("volume extent in mm", {mGeometry.volExtent.sliceWidth, mGeometry.volExtent.sliceHeight,
                                              mGeometry.volExtent.volDepth});
  printVector<double>("x,y coordinates of first voxel in mm", {mHeader.volOffset.x, mHeader.volOffset.y});
  printValue("volume offset in z in mm", mHeader.volOffset.z);
  printValue("number of time frames", mHeader.nFrames);
  printValue("number of voxels per frame", mGeometry.nVoxelsPerFrame);
  printValue("total number of voxels", mGeometry.nVoxelsTotal);
  printEmptyLine();
}

void VolData::checkNFrames(int nFrames) const
{
  if (mHeader.nFrames != nFrames)
  {
    error("Wrong number of frames (expected ", nFrames, ")");
  }
}

void VolData::assign(const VolData& vol)
{
  if (!isAllocated())
  {
    error("Volume not allocated");
  }
  if (mHeader != vol.mHeader || mHeader.nFrames != vol.mHeader.nFrames)
  {
    error("Volume assigned is not the right size");
  }
  std::copy(vol.mData.begin(), vol.mData.end(), mData.begin());
}

void VolData::assignFrame(const VolData& vol, int frame)
{
  if (!isAllocated())
  {
    error("Volume not allocated");
  }
  if (mHeader != vol.mHeader)
  {
    error("Volume assigned is not the right size");
  }
  const float* src = vol.mData.data() + static_cast<size_t>(frame) * mGeometry.nVoxelsPerFrame;
  std::copy(src, src + mGeometry.nVoxelsPerFrame, mActive);
}

void VolData::setAllVoxels(types::VoxelValue v)
{
  if (!isAllocated())
  {
    error("Volume not allocated");
  }
  std::fill(mActive, mActive + mGeometry.nVoxelsPerFrame, v);
}

void VolData::setAllVoxelsAllFrames(types::VoxelValue v)
{
  if (!isAllocated())
  {
    error("Volume not allocated");
  }
  std::fill(mData.begin(), mData.end(), v);
}

VolData& VolData::operator*=(const VolData& in)
{
  for (int i = 0; i < mGeometry.nVoxelsPerFrame; ++i)
  {
    mActive[i] = (mActive[i] > EPSILON && in.mActive[i] > EPSILON) ? mActive[i] * in.mActive[i] : 0.0f;
  }
  return *this;
}

VolData& VolData::operator/=(const VolData& in)
{
  for (int i = 0; i < mGeometry.nVoxelsPerFrame; ++i)
  {
    mActive[i] = (mActive[i] > EPSILON && in.mActive[i] > EPSILON) ? mActive[i] / in.mActive[i] : 0.0f;
  }
  return *this;
}

void VolData::setActiveFrame(int frame) const
{
  if (!(frame >= 0 && frame < mHeader.nFrames))
  {
    error("Invalid frame");
  }
  mActiveFrame = frame;
  mActive = const_cast<float*>(mData.data()) + static_cast<size_t>(frame) * mGeometry.nVoxelsPerFrame;
}

types::VoxelValue VolData::computeLineIntegral(types::PathElement* path) const
{
  types::VoxelValue line = 0.0f;
  for (int k = 0; path[k].coord != -1; ++k)
  {
    line = static_cast<float>(static_cast<double>(line) + path[k].length * static_cast<double>(mActive[path[k].coord]));
  }
  return line;
}

void VolData::projectLineIntegral(types::PathElement* path, types::VoxelValue line)
{
  for (int k = 0; path[k].coord != -1; ++k)
  {
    float& v = mActive[path[k].coord];
    v = static_cast<float>(static_cast<double>(v) + path[k].length * static_cast<double>(line));
  }
}
