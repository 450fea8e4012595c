// Sinogram data model and its Interfile I/O (.hs header + raw float32 .s),
// with the behaviour of FIR's ProjHeader/ProjData/ProjInterfileReader
// (src_lib/ProjHeader.cc, ProjData.cc, ProjInterfileReader.cc).  Header
// validation and ProjGeometry come from the C ABI; the bin-wise arithmetic
// runs on the GPU.
#include <KeyParser.h>
#include <ProjData.h>
#include <console.h>
#include <fir_cuda.h>
#include <macros.h>
#include <runtime.h>

#include <algorithm>
#include <filesystem>
#include <fstream>

void ProjHeader::setDefaults()
{
  nRings = 0;
  nCrystalsPerRing = 0;
  segmentSpan = 1;
  nSegments = 1;
  nTangCoords = 0;
}

void ProjHeader::check()
{
  const fir_proj_desc d{nRings, nCrystalsPerRing, segmentSpan, nSegments, nTangCoords};
  fir_proj_info info;
  if (fir_proj_geometry(&d, &info, nullptr) != FIR_OK)
  {
    error(fir_last_error());
  }
  nTangCoords = info.n_tang_coords;
}

void ProjGeometry::fill(const ProjHeader& h)
{
  const fir_proj_desc d{h.nRings, h.nCrystalsPerRing, h.segmentSpan, h.nSegments, h.nTangCoords};
  fir_proj_info info;
  nAxialCoords.assign(static_cast<size_t>(std::max(h.nSegments, 0)), 0);
  if (fir_proj_geometry(&d, &info, nAxialCoords.data()) != FIR_OK)
  {
    error(fir_last_error());
  }
  nBins = static_cast<int>(info.n_bins);
  segOffset = info.seg_offset;
  tangCoordOffset = info.tang_offset;
  nViews = info.n_views;
  halfSegmentSpan = info.half_span;
  maxRingDiff = info.max_ring_diff;
}

ProjData::ProjData() { mHeader.setDefaults(); }

ProjData::ProjData(const std::string& file, ConstructionMode mode, types::BinValue init) : ProjData()
{
  read(file, mode, init);
}

ProjData::ProjData(const ProjData& proj, ConstructionMode mode, types::BinValue init) : ProjData()
{
  copy(proj, mode, init);
}

void ProjData::allocate(bool initialize, types::BinValue initValue)
{
  mData.assign(static_cast<size_t>(mGeometry.nBins), initialize ? initValue : 0.0f);
  mSegments.assign(static_cast<size_t>(mHeader.nSegments), nullptr);
  size_t off = 0;
  for (int seg = -mGeometry.segOffset; seg <= mGeometry.segOffset; ++seg)
  {
    mSegments[seg + mGeometry.segOffset] = mData.data() + off;
    off += static_cast<size_t>(mGeometry.getNAxialCoords(seg)) * mGeometry.nViews * mHeader.nTangCoords;
  }
}

void ProjData::read(const std::string& headerFile, ConstructionMode mode, types::BinValue initValue)
{
  std::string dataFile;
  ProjHeader h;
  h.setDefaults();
  KeyParser kp;
  kp.addStartKey("!PROJECTION DATA PARAMETERS");
  kp.addKey("name of data file", &dataFile);
  kp.addKey("number of rings", &h.nRings);
  kp.addKey("number of crystals per ring", &h.nCrystalsPerRing);
  kp.addKey("segment span", &h.segmentSpan);
  kp.addKey("number of segments", &h.nSegments);
  kp.addKey("number of tangential coordinates", &h.nTangCoords);
  kp.addStopKey("!END OF PROJECTION DATA PARAMETERS");
  kp.parse(headerFile);
  if (!dataFile.empty() && dataFile[0] != '/')
  {
    const auto slash = headerFile.find_last_of('/');
    if (slash != std::string::npos)
    {
      dataFile.insert(0, headerFile, 0, slash + 1);
    }
  }
  h.check();
  mHeader = h;
  mGeometry.fill(mHeader);
  allocate(mode == ConstructionMode::INITIALIZE, initValue);
  if (mode != ConstructionMode::READ_DATA)
  {
    return;
  }
  std::ifstream in(dataFile, std::ios::binary);
  if (!in.is_open())
  {
    error("Couldn't open file ", dataFile);
  }
  in.read(reinterpret_cast<char*>(mData.data()), static_cast<std::streamsize>(mData.size() * sizeof(float)));
  if (!in)
  {
    error("The number of bins that were read from the data file (", in.gcount(),
          ") is inferior to that expected from the header file (", mGeometry.nBins, ")");
  }
}

void ProjData::copy(const ProjData& proj, ConstructionMode mode, types::BinValue initValue)
{
  mHeader = proj.mHeader;
  mGeometry = proj.mGeometry;
  allocate(mode == ConstructionMode::INITIALIZE, initValue);
  if (mode == ConstructionMode::READ_DATA)
  {
    std::copy(proj.mData.begin(), proj.mData.end(), mData.begin());
  }
}

void ProjData::write(const std::string& outputProjFile) const
{
  if (mData.empty())
  {
    error("Projection data is not allocated");
  }
  std::filesystem::path hdr(outputProjFile), dat(outputProjFile);
  hdr.replace_extension(".hs");
  dat.replace_extension(".s");
  std::ofstream os(hdr);
  if (!os.is_open())
  {
    error("Couldn't create file ", hdr.string());
  }
  // ProjInterfileReader.cc:187-242
  os << "!PROJECTION DATA PARAMETERS :=\n";
  os << "name of data file := " << dat.filename().string() << "\n";
  os << "number of rings := " << mHeader.nRings << "\n";
  os << "number of crystals per ring := " << mHeader.nCrystalsPerRing << "\n";
  os << "segment span := " << mHeader.segmentSpan << "\n";
  os << "number of segments := " << mHeader.nSegments << "\n";
  os << "number of tangential coordinates := " << mHeader.nTangCoords << "\n";
  os << "!END OF PROJECTION DATA PARAMETERS :=\n";
  std::ofstream ds(dat, std::ios::binary);
  if (!ds.is_open())
  {
    error("Couldn't create file ", dat.string());
  }
  ds.write(reinterpret_cast<const char*>(mData.data()), static_cast<std::streamsize>(mData.size() * sizeof(float)));
}

void ProjData::printContent() const
{
  echo("= Projection header:");
  printEmptyLine();
  printValue("number of rings", mHeader.nRings);
  printValue("number of crystals per ring", mHeader.nCrystalsPerRing);
  printValue("segment span", mHeader.segmentSpan);
  printValue("number of segments", mHeader.nSegments);
  printVector("number of axial coords", mGeometry.nAxialCoords);
  printValue("number of views", mGeometry.nViews);
  printValue("number of tangential coordinates", mHeader.nTangCoords);
  printValue("total number of bins", mGeometry.nBins);
  printValue("segment offset", mGeometry.segOffset);
  printValue("tangential coordinate offset", mGeometry.tangCoordOffset);
  printValue("half the segment span", mGeometry.halfSegmentSpan);
  printValue("maximum ring difference", mGeometry.maxRingDiff);
  printEmptyLine();
}

void ProjData::checkNSubsets(int nSubsets) const
{
  if (nSubsets <= 0 || mGeometry.nViews % nSubsets != 0)
  {
    error("Number of subsets must be a divisor of ", mGeometry.nViews);
  }
}

void ProjData::setAllBins(types::BinValue value)
{
  if (mData.empty())
  {
    error("Projection not allocated");
  }
  std::fill(mData.begin(), mData.end(), value);
}

std::tuple<int, int> ProjData::getCrystalAxialCoord(int seg, int axial) const
{
  // ProjData.cc:198-299
  if (mHeader.segmentSpan == 1)
  {
    if (seg == 0)
    {
      return {2 * axial, 2 * axial};
    }
    return seg > 0 ? std::tuple<int, int>{2 * (axial + seg), 2 * axial}
                   : std::tuple<int, int>{2 * axial, 2 * (axial - seg)};
  }
  if (seg == 0)
  {
    return {axial, axial};
  }
  const int mid = ABS(seg) * mHeader.segmentSpan;
  const int h = mGeometry.halfSegmentSpan;
  if (axial < h)
  {
    const int rd = mid - h + axial;
    return seg > 0 ? std::tuple<int, int>{2 * rd, 0} : std::tuple<int, int>{0, 2 * rd};
  }
  const int inv = mGeometry.getNAxialCoords(seg) - axial - 1;
  if (inv < h)
  {
    const int rd = mid - h + inv;
    const int smax = 2 * mHeader.nRings - 2;
    return seg > 0 ? std::tuple<int, int>{smax, smax - 2 * rd} : std::tuple<int, int>{smax - 2 * rd, smax};
  }
  const int adj = axial - h;
  return seg > 0 ? std::tuple<int, int>{2 * mid + adj, adj} : std::tuple<int, int>{adj, 2 * mid + adj};
}

std::tuple<int, int> ProjData::getCrystalAngCoord(int view, int tang) const
{
  // ProjData.cc:301-340
  const int shift = tang >= 0 ? tang / 2 : (tang - 1) / 2;
  const int odd = ABS(tang) % 2;
  const int n = mHeader.nCrystalsPerRing;
  int a = view + shift + odd;
  int b = view + mGeometry.nViews - shift;
  if (a < 0)
    a += n;
  else if (a >= n)
    a -= n;
  if (b < 0)
    b += n;
  else if (b >= n)
    b -= n;
  return {a, b};
}

ProjData& ProjData::operator*=(const ProjData& in)
{
  if (!(mHeader == in.mHeader))
  {
    error("Projections multiplied do not have the same header");
  }
  const fir_proj_desc d = fir_runtime::projDesc(*this);
  fir_runtime::check(fir_proj_multiply(fir_runtime::context(), &d, mData.data(), in.mData.data()), "ProjData *=");
  return *this;
}

void ProjData::exponential()
{
  const fir_proj_desc d = fir_runtime::projDesc(*this);
  fir_runtime::check(fir_proj_exponential(fir_runtime::context(), &d, mData.data()), "ProjData::exponential");
}

bool ProjData::getBinCoordinates(int crystalAxialCoord1, int crystalAngCoord1, int crystalAxialCoord2,
                                 int crystalAngCoord2, int* seg, int* view, int* axialCoord, int* tangCoord) const
{
  const fir_proj_desc d = fir_runtime::projDesc(*this);
  const int pair[4] = {crystalAxialCoord1, crystalAngCoord1, crystalAxialCoord2, crystalAngCoord2};
  int coords[5] = {0, 0, 0, 0, 0};
  fir_runtime::check(fir_bin_coordinates(fir_runtime::context(), &d, 1, pair, coords, nullptr),
                     "ProjData::getBinCoordinates");
  if (coords[0] == 0)
  {
    return false;
  }
  *seg = coords[1];
  *view = coords[2];
  *axialCoord = coords[3];
  *tangCoord = coords[4];
  return true;
}

void ProjData::rebinWeight()
{
  const fir_proj_desc d = fir_runtime::projDesc(*this);
  fir_runtime::check(fir_proj_rebin_weight(fir_runtime::context(), &d, mData.data()), "ProjData::rebinWeight");
}
