// C ABI of the B200 path (include/fir_cuda.h): validation, contexts, host
// staging, geometry tables and launch orchestration.  The kernels live in
// projector.cu, image_ops.cu, frames.cu, deterministic.cu and batch.cu; the
// batched OSEM's ABI in capi_batch.cu; shared declarations in
// capi_common.h.
//
// Validation reproduces the checks FIR performs before it projects, with
// FIR's messages:
//   ProjHeader::check             src_lib/ProjHeader.cc:6-106
//   ProjGeometry::fill            src_lib/ProjHeader.cc:108-186
//   ScannerHeader::check          src_lib/ScannerHeader.cc:26-303
//   ScannerGeometry::fill         src_lib/ScannerHeader.cc:305-342
//   VolHeader::check              src_lib/VolHeader.cc:5-29
//   ScannerData::checkProjData    src_lib/ScannerData.cc:31-44
//   ProjData::checkNSubsets       src_lib/ProjData.cc:166-174
//   VolData::checkNFrames         src_lib/VolData.cc:227-233
#include "capi_common.h"

#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace fir::abi
{
thread_local std::string g_error;

void cuda_ok(cudaError_t e, const char* what)
{
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
    {
      fail(FIR_ERR_OUT_OF_MEMORY, what, ": ", cudaGetErrorString(e));
    }
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    {
      fail(FIR_ERR_NO_DEVICE, what, ": ", cudaGetErrorString(e));
    }
    fail(FIR_ERR_CUDA, what, ": ", cudaGetErrorString(e));
  }
}

// ------------------------------------------------------------ geometry


ProjInfo check_proj(const fir_proj_desc* desc)
{
  if (desc == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "projection descriptor is NULL");
  }
  ProjInfo p;
  p.d = *desc;
  auto& h = p.d;
  if (h.n_rings <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of rings\" must be provided and > 0");
  }
  if (h.n_crystals_per_ring <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of crystals per ring\" must be provided and > 0");
  }
  if (h.n_crystals_per_ring % 4 != 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of crystals per ring\" must be a multiple of four");
  }
  if (h.segment_span <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"segment span\" must be > 0");
  }
  if (h.segment_span % 2 != 1)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"segment span\" must be an odd number");
  }
  const int max_span = 2 * h.n_rings - 1;
  if (h.segment_span > max_span)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "For ", h.n_rings, " ring(s), \"segment span\" must not be > ", max_span);
  }
  if (h.n_segments < 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of segments\" must not be negative");
  }
  if (h.n_segments % 2 != 1)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of segments\" must be an odd number");
  }
  int max_nseg = max_span / h.segment_span;
  max_nseg -= 1 - max_nseg % 2;
  if (h.n_segments > max_nseg)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "For ", h.n_rings, " ring(s) and a segment span of ", h.segment_span,
         ", \"number of segments\" must not be > ", max_nseg);
  }
  if (h.n_tang_coords < 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"number of tangential coordinates\" must not be negative");
  }
  const int max_tang = h.n_crystals_per_ring - 1;
  if (h.n_tang_coords == 0)
  {
    h.n_tang_coords = max_tang;
  }
  else if (h.n_tang_coords > max_tang)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "For ", h.n_crystals_per_ring,
         " crystals per ring, \"number of tangential coordinates\" must not be > ", max_tang);
  }
  if (h.n_segments > kMaxSegments)
  {
    fail(FIR_ERR_NOT_SUPPORTED, "at most ", kMaxSegments, " segments are supported");
  }
  // ProjGeometry::fill
  auto& g = p.g;
  g.seg_offset = (h.n_segments - 1) / 2;
  g.tang_offset = h.n_tang_coords / 2;
  g.n_tang_coords = h.n_tang_coords;
  p.n_axial.resize(h.n_segments);
  for (int seg = -g.seg_offset; seg <= g.seg_offset; ++seg)
  {
    const int a = seg < 0 ? -seg : seg;
    int len;
    if (h.segment_span == 1)
    {
      len = h.n_rings - a;
    }
    else
    {
      len = 2 * h.n_rings - 1;
      if (a >= 1)
      {
        len -= h.segment_span + 1;
      }
      if (a >= 2)
      {
        len -= 2 * h.segment_span * (a - 1);
      }
    }
    p.n_axial[seg + g.seg_offset] = len;
  }
  g.n_views = h.n_crystals_per_ring / 2;
  g.n_bins = 0;
  for (int len : p.n_axial)
  {
    g.n_bins += (long long)len * g.n_views * h.n_tang_coords;
  }
  g.half_span = (h.segment_span - 1) / 2;
  g.max_ring_diff = h.segment_span == 1 ? g.seg_offset
                                         : g.half_span + (g.seg_offset > 0 ? g.seg_offset * h.segment_span : 0);
  if (g.n_bins > 0x7fffffffLL)
  {
    // FIR counts bins in int (ProjHeader.h:45)
    fail(FIR_ERR_NOT_SUPPORTED, "total number of bins ", g.n_bins, " exceeds 2^31-1");
  }
  return p;
}


ScannerInfo scanner_tables(const fir_scanner_desc* d0, bool tables)
{
  if (d0 == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "scanner descriptor is NULL");
  }
  fir_scanner_desc s = *d0;
  for (int i = 0; i < 3; ++i)
  {
    if (s.crystal_dims[i] < 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"crystal dimensions XYZ in mm\" must not be negative");
    }
  }
  if (s.crystal_repeat[0] <= 0 || s.crystal_repeat[1] <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"crystal repeat numbers YZ\" must be > 0");
  }
  if (s.inter_crystal[0] < 0 || s.inter_crystal[1] < 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"inter-crystal distance YZ in mm\" must not be negative");
  }
  for (int i = 0; i < 3; ++i)
  {
    if (s.module_dims[i] < 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"module dimensions XYZ in mm\" must not be negative");
    }
  }
  if (s.module_repeat[0] <= 0 || s.module_repeat[1] <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"module repeat numbers YZ\" must be > 0");
  }
  if (s.inter_module[0] < 0 || s.inter_module[1] < 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"inter-module distance YZ in mm\" must not be negative");
  }
  for (int i = 0; i < 3; ++i)
  {
    if (s.rsector_dims[i] < 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "Elements of \"rSector dimensions XYZ in mm\" must not be negative");
    }
  }
  if (s.rsector_repeat <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"rSector repeat number\" must be present and > 0");
  }
  if (s.rsector_inner_radius <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "\"rSector inner radius in mm\" must be present and > 0");
  }
  if (s.crystal_repeat[0] > 1 && s.crystal_dims[1] == 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Crystal repeat number in Y cannot be > 1 if crystal dimension in Y is zero");
  }
  if (s.crystal_repeat[1] > 1 && s.crystal_dims[2] == 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Crystal repeat number in Z cannot be > 1 if crystal dimension in Z is zero");
  }
  const double min_mod[3] = {
    s.crystal_dims[0],
    s.crystal_dims[1] * s.crystal_repeat[0] + s.inter_crystal[0] * (s.crystal_repeat[0] - 1),
    s.crystal_dims[2] * s.crystal_repeat[1] + s.inter_crystal[1] * (s.crystal_repeat[1] - 1)};
  const char* axis = "XYZ";
  for (int i = 0; i < 3; ++i)
  {
    if (s.module_dims[i] == 0.0)
    {
      s.module_dims[i] = min_mod[i];
    }
    else if (s.module_dims[i] < min_mod[i])
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "Module dimension in ", axis[i], " must be >= ", min_mod[i]);
    }
  }
  if (s.module_repeat[0] > 1 && s.module_dims[1] == 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Module repeat number in Y cannot be > 1 if module dimension in Y is zero");
  }
  if (s.module_repeat[1] > 1 && s.module_dims[2] == 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Module repeat number in Z cannot be > 1 if module dimension in Z is zero");
  }
  const double min_rs[3] = {
    s.module_dims[0],
    s.module_dims[1] * s.module_repeat[0] + s.inter_module[0] * (s.module_repeat[0] - 1),
    s.module_dims[2] * s.module_repeat[1] + s.inter_module[1] * (s.module_repeat[1] - 1)};
  for (int i = 0; i < 3; ++i)
  {
    if (s.rsector_dims[i] == 0)
    {
      s.rsector_dims[i] = min_rs[i];
    }
    else if (s.rsector_dims[i] < min_rs[i])
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "rSector dimension in ", axis[i], " must be >= ", min_rs[i]);
    }
  }
  ScannerInfo out;
  out.n_cpr = s.crystal_repeat[0] * s.module_repeat[0] * s.rsector_repeat;
  out.n_rings = s.crystal_repeat[1] * s.module_repeat[1];
  if (!tables)
  {
    return out;
  }
  // ScannerData::computeCrystalXYPositionVector (ScannerData.cc:248-329):
  // the first rSector is vertical at x = inner radius + depth/2 and is
  // repeated by rotation; crystal 0 is the middle crystal of rSector 0.
  const double cvy = s.crystal_dims[1] + s.inter_crystal[0];
  const double cvz = s.crystal_dims[2] + s.inter_crystal[1];
  const double mvy = s.module_dims[1] + s.inter_module[0];
  const double mvz = s.module_dims[2] + s.inter_module[1];
  const double tx = s.rsector_inner_radius + s.rsector_dims[0] / 2;
  const int crystal_offset = s.module_repeat[0] * s.crystal_repeat[0] / 2;
  const int ncy = s.crystal_repeat[0], nmy = s.module_repeat[0];
  const double first_y = -((nmy - 1) * mvy + (ncy - 1) * cvy) / 2.0;
  const int nrs = nmy * ncy;
  std::vector<double> rsy(nrs);
  for (int m = 0; m < nmy; ++m)
  {
    for (int c = 0; c < ncy; ++c)
    {
      rsy[m * ncy + c] = m * mvy + c * cvy + first_y;
    }
  }
  const double angle_interval = 2 * 3.141592653589793 / s.rsector_repeat;
  const int first_index = out.n_cpr - crystal_offset;
  out.xy.resize(2 * (size_t)out.n_cpr);
  for (int i = 0; i < first_index; ++i)
  {
    const double x = tx;
    const int io = i + crystal_offset;
    const double y = rsy[io % nrs];
    const double angle = (io / nrs) * angle_interval;
    const double ca = std::cos(angle);
    const double sa = std::sin(angle);
    out.xy[2 * i] = x * ca - y * sa;
    out.xy[2 * i + 1] = x * sa + y * ca;
  }
  for (int i = first_index; i < out.n_cpr; ++i)
  {
    out.xy[2 * i] = tx;
    out.xy[2 * i + 1] = rsy[i - first_index];
  }
  // computeSliceZPositionVector (ScannerData.cc:331-377): even slices on the
  // rings, odd slices half-way between neighbouring rings.
  const int ncz = s.crystal_repeat[1], nmz = s.module_repeat[1];
  const double first_z = -((nmz - 1) * mvz + (ncz - 1) * cvz) / 2.0;
  std::vector<double> ringz(nmz * ncz);
  for (int m = 0; m < nmz; ++m)
  {
    for (int c = 0; c < ncz; ++c)
    {
      ringz[m * ncz + c] = m * mvz + c * cvz + first_z;
    }
  }
  out.z.resize(2 * (size_t)out.n_rings - 1);
  for (int k = 0; k < 2 * out.n_rings - 1; ++k)
  {
    out.z[k] = k % 2 == 0 ? ringz[k / 2] : (ringz[k / 2] + ringz[(k + 1) / 2]) / 2.0;
  }
  return out;
}


VolInfo check_vol(const fir_vol_desc* v)
{
  if (v == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "volume descriptor is NULL");
  }
  if (v->nx <= 0 || v->ny <= 0 || v->nz <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Number of voxels must be greater than zero in each dimension");
  }
  if (!(v->voxel_x > 0) || !(v->voxel_y > 0) || !(v->voxel_z > 0))
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Voxel extent must be greater than zero in each dimension");
  }
  if (v->n_frames <= 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Number of frames must be greater than zero");
  }
  VolInfo out{*v, (long long)v->nx * v->ny * v->nz};
  if (out.nvox > 0x7fffffffLL)
  {
    // FIR indexes voxels with int (types.h:7-8)
    fail(FIR_ERR_NOT_SUPPORTED, "volume of ", out.nvox, " voxels exceeds 2^31-1");
  }
  return out;
}

void check_frames(const VolInfo& v, int n)
{
  if (v.d.n_frames != n)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Wrong number of frames (expected ", n, ")");
  }
}

void check_subsets(const ProjInfo& p, int n_subsets)
{
  if (n_subsets <= 0 || p.g.n_views % n_subsets != 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Number of subsets must be a divisor of ", p.g.n_views);
  }
}

}  // namespace fir::abi

// ------------------------------------------------------------ context



namespace fir::abi
{
fir_ctx& check_ctx(fir_ctx* c)
{
  if (c == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "context is NULL");
  }
  cuda_ok(cudaSetDevice(c->device), "cudaSetDevice");
  return *c;
}

LaunchCfg cfg_of(fir_ctx& c)
{
  return LaunchCfg{c.block, c.stream, static_cast<int*>(c.check.p)};
}

void after_launch(fir_ctx& c, int n = 1)
{
  c.launches += n;
  cuda_ok(cudaGetLastError(), "kernel launch");
}

cudaEvent_t take_event(fir_ctx& c)
{
  if (!c.ev_pool.empty())
  {
    cudaEvent_t e = c.ev_pool.back();
    c.ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cuda_ok(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

// Brackets one projector-kernel launch with events when timing is on.
template<typename F>
void timed_launch(fir_ctx& c, F&& launch)
{
  if (!c.timing)
  {
    launch();
    after_launch(c);
    return;
  }
  cudaEvent_t a = take_event(c), b = take_event(c);
  cuda_ok(cudaEventRecord(a, c.stream), "cudaEventRecord");
  launch();
  after_launch(c);
  cuda_ok(cudaEventRecord(b, c.stream), "cudaEventRecord");
  c.ev_pending.emplace_back(a, b);
}

void drain_timing(fir_ctx& c)
{
  for (auto& p : c.ev_pending)
  {
    cuda_ok(cudaEventSynchronize(p.second), "cudaEventSynchronize");
    float ms = 0.0f;
    cuda_ok(cudaEventElapsedTime(&ms, p.first, p.second), "cudaEventElapsedTime");
    c.timed_ms += ms;
    c.timed_n += 1;
    c.ev_pool.push_back(p.first);
    c.ev_pool.push_back(p.second);
  }
  c.ev_pending.clear();
}

// Deterministic-mode backprojection of vals (per bin, or per enumerated LOR
// when by_enum) into img, FIR's serial order; scratch from the context.
void det_backproject(fir_ctx& c, const Grid& g, const Sino& s, const Tables& t, const float* vals, bool by_enum,
                     float* img, long long nvox, const int* counts = nullptr)
{
  const ScratchFn scratch = [&c](int slot, size_t bytes) -> void* {
    DevBuf& b = slot == 0 ? c.det : c.det_pairs;
    try
    {
      return b.ensure(bytes);
    }
    catch (const Failure&)
    {
      return nullptr;
    }
  };
  long long launches = 0;
  // chunks of at most det_chunk pairs (default 2^28: about 6 GiB of keys,
  // products and sort buffers)
  cuda_ok(deterministic_backproject(g, s, t, vals, by_enum, counts, img, scratch, c.det_chunk, nvox, cfg_of(c),
                                    &launches),
          "deterministic backprojection");
  c.launches += launches;
}

// Double copy of a float image in context scratch, for the projector gathers.
const double* widen(fir_ctx& c, const float* img, long long n)
{
  double* d = static_cast<double*>(c.wide.ensure((size_t)n * sizeof(double)));
  launch_widen(n, img, d, cfg_of(c));
  after_launch(c);
  return d;
}

// Double copies of a float image for a projection: with x and y exchanged
// too while both fit in L2 (use_exchanged).
struct Widened
{
  const double* img;
  const double* img_t;  // null: one orientation
};

Widened widen_for_projection(fir_ctx& c, const Grid& g, const float* img)
{
  const long long n = (long long)g.nxy * g.nz;
  if (!use_exchanged(c, g, 16.0))
  {
    return Widened{widen(c, img, n), nullptr};
  }
  double* d = static_cast<double*>(c.wide.ensure((size_t)n * sizeof(double)));
  double* d_t = static_cast<double*>(c.wide_t.ensure((size_t)n * sizeof(double)));
  launch_widen_oriented(g.nx, g.ny, g.nz, img, d, d_t, cfg_of(c));
  after_launch(c);
  return Widened{d, d_t};
}

// s with the compacted list of its bins whose measured value is not 0
// (FIR_OPT_SKIP_ZERO_BINS), built on the context stream in context scratch.
Sino nonzero_bins(fir_ctx& c, const Sino& s, const float* sino)
{
  size_t temp = 0;
  cuda_ok(launch_nonzero_list(s, sino, nullptr, nullptr, nullptr, &temp, cfg_of(c)), "cub::DeviceSelect");
  const size_t list_bytes = ((size_t)s.n_enum * sizeof(int) + 255) / 256 * 256;
  auto* base = static_cast<unsigned char*>(c.compact.ensure(list_bytes + 256 + temp));
  int* list = reinterpret_cast<int*>(base);
  int* count = reinterpret_cast<int*>(base + list_bytes);
  cuda_ok(launch_nonzero_list(s, sino, list, count, base + list_bytes + 256, &temp, cfg_of(c)),
          "cub::DeviceSelect");
  after_launch(c);
  Sino out = s;
  out.list = list;
  out.list_n = count;
  return out;
}

// img += backprojection of sino (nullptr: all ones) over the subset of s, in
// the atomic mode; LORs running mostly along x accumulate in an x/y-exchanged
// scratch image that is added into img afterwards, while both fit in L2.
void backproject_subset(fir_ctx& c, const Grid& g, const Sino& s, const Tables& t, const float* sino, float* img,
                        bool skip_zero)
{
  float* img_t = nullptr;
  const long long n = (long long)g.nxy * g.nz;
  if (use_exchanged(c, g, 8.0))
  {
    img_t = static_cast<float*>(c.bp_t.ensure((size_t)n * sizeof(float)));
    cuda_ok(cudaMemsetAsync(img_t, 0, (size_t)n * sizeof(float), c.stream), "cudaMemsetAsync");
  }
  // skipped bins: listed out of the enumeration
  const Sino sl = skip_zero && sino != nullptr && s.n_enum > 0 ? nonzero_bins(c, s, sino) : s;
  timed_launch(c, [&] { launch_backward(g, sl, t, sino, img, img_t, skip_zero, cfg_of(c)); });
  if (img_t != nullptr)
  {
    launch_merge_oriented(g.nx, g.ny, g.nz, img, img_t, cfg_of(c));
    after_launch(c);
  }
}

// bp (zeroed by the caller) += backprojection of sino / (projection of img +
// bias) over the subset of s: the fused kernel, or in deterministic mode the
// ratio kernel followed by the ordered scatter.  The fused kernel reads and
// accumulates LORs that run mostly along x in images with x and y exchanged
// (double copy and accumulator in context scratch); the accumulator is added
// back into bp after the kernel, or, with defer_merge, returned (null: none)
// for the caller to add (launch_em_update_oriented).
const float* ratio_backproject(fir_ctx& c, const Grid& g, const Sino& s_all, const Tables& t, const float* img,
                               const float* sino, const float* mult, const float* bias, float* bp, long long nvox,
                               bool defer_merge = false)
{
  // skipped bins: listed out of the atomic kernels' enumeration
  const bool listed = c.skip_zero != 0 && c.backproj == FIR_BACKPROJ_ATOMIC && s_all.n_enum > 0;
  const Sino s = listed ? nonzero_bins(c, s_all, sino) : s_all;
  if (c.traversal == FIR_TRAVERSAL_FLOAT && c.backproj == FIR_BACKPROJ_ATOMIC && mult == nullptr &&
      c.step_limit == 0)
  {
    // the opt-in float loop: float images in both orientations while they
    // and the accumulators fit in L2 (16 B per voxel)
    const size_t n = (size_t)nvox;
    float* img_t = nullptr;
    float* bp_t = nullptr;
    if (use_exchanged(c, g, 16.0))
    {
      img_t = static_cast<float*>(c.img_t.ensure(n * sizeof(float)));
      bp_t = static_cast<float*>(c.bp_t.ensure(n * sizeof(float)));
      cuda_ok(cudaMemsetAsync(bp_t, 0, n * sizeof(float), c.stream), "cudaMemsetAsync");
      launch_exchange_float(g.nx, g.ny, g.nz, img, img_t, cfg_of(c));
      after_launch(c);
    }
    timed_launch(c, [&] {
      launch_osem_subset_float(g, s, t, img, img_t, sino, bias, bp, bp_t, c.skip_zero != 0, cfg_of(c));
    });
    if (bp_t != nullptr && defer_merge)
    {
      return bp_t;
    }
    if (bp_t != nullptr)
    {
      launch_merge_oriented(g.nx, g.ny, g.nz, bp, bp_t, cfg_of(c));
      after_launch(c);
    }
    return nullptr;
  }
  if (c.backproj == FIR_BACKPROJ_DETERMINISTIC)
  {
    const double* wimg = widen(c, img, nvox);
    // the ratio and, from the same walks, the pair count of every LOR
    const size_t ne = (size_t)std::max(s.n_enum, 1);
    float* ratio = static_cast<float*>(c.ratio.ensure(ne * (sizeof(float) + sizeof(int))));
    int* counts = reinterpret_cast<int*>(ratio + ne);
    timed_launch(c, [&] { launch_ratio(g, s, t, wimg, sino, mult, bias, ratio, counts, cfg_of(c)); });
    det_backproject(c, g, s, t, ratio, true, bp, nvox, counts);
    return nullptr;
  }
  if (!use_exchanged(c, g))
  {
    if (!use_exchanged(c, g, 12.0) && use_exchanged(c, g, 8.0))
    {
      // the double copy and the accumulator (12 B/voxel) overflow L2, the
      // float image and the accumulator (8 B/voxel) fit: gather floats, one
      // launch per orientation, each with its own image and accumulator
      const size_t n = (size_t)nvox;
      float* img_t = static_cast<float*>(c.img_t.ensure(n * sizeof(float)));
      float* bp_t = static_cast<float*>(c.bp_t.ensure(n * sizeof(float)));
      cuda_ok(cudaMemsetAsync(bp_t, 0, n * sizeof(float), c.stream), "cudaMemsetAsync");
      launch_exchange_float(g.nx, g.ny, g.nz, img, img_t, cfg_of(c));
      after_launch(c);
      timed_launch(c, [&] {
        launch_osem_subset_float_image(g, s, t, img, img_t, sino, mult, bias, bp, bp_t, c.skip_zero != 0,
                                       cfg_of(c));
      });
      if (defer_merge)
      {
        return bp_t;
      }
      launch_merge_oriented(g.nx, g.ny, g.nz, bp, bp_t, cfg_of(c));
      after_launch(c);
      return nullptr;
    }
    const double* wimg = widen(c, img, nvox);
    timed_launch(c, [&] {
      launch_osem_subset(g, s, t, wimg, nullptr, sino, mult, bias, bp, nullptr, c.skip_zero != 0, cfg_of(c));
    });
    return nullptr;
  }
  const size_t n = (size_t)nvox;
  double* wimg = static_cast<double*>(c.wide.ensure(n * sizeof(double)));
  double* wimg_t = static_cast<double*>(c.wide_t.ensure(n * sizeof(double)));
  float* bp_t = static_cast<float*>(c.bp_t.ensure(n * sizeof(float)));
  cuda_ok(cudaMemsetAsync(bp_t, 0, n * sizeof(float), c.stream), "cudaMemsetAsync");
  launch_widen_oriented(g.nx, g.ny, g.nz, img, wimg, wimg_t, cfg_of(c));
  after_launch(c);
  timed_launch(c, [&] {
    launch_osem_subset(g, s, t, wimg, wimg_t, sino, mult, bias, bp, bp_t, c.skip_zero != 0, cfg_of(c));
  });
  if (defer_merge)
  {
    return bp_t;
  }
  launch_merge_oriented(g.nx, g.ny, g.nz, bp, bp_t, cfg_of(c));
  after_launch(c);
  return nullptr;
}

Tables tables_of(fir_ctx& c, const ProjInfo& p)
{
  if (!c.have_scanner)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "no scanner set on the context (fir_ctx_set_scanner)");
  }
  if (p.d.n_rings != c.scan_rings || p.d.n_crystals_per_ring != c.scan_cpr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Projection must have the same number of rings (", c.scan_rings,
         ") and the same number of crystals per ring (", c.scan_cpr, ") as the scanner");
  }
  return Tables{static_cast<const double2*>(c.xy.p), static_cast<const double*>(c.z.p)};
}

// The exchanged images halve the cache lines a warp's gathers and atomics
// touch, but double the image bytes in use.  With both orientations in L2
// they pay (clinical 200x200x64 volume: subset kernel 2.36 -> 2.09 ms); a
// 320x320x128 volume (315 MB for both) ran 4 % slower with them.
bool use_exchanged(fir_ctx& c, const Grid& g, double bytes_per_voxel)
{
  if ((g.ny + 31) / 32 > 65535)
  {
    return false;  // beyond the tile grid of the exchange kernels
  }
  if (c.l2_bytes == 0)
  {
    int v = 0;
    cuda_ok(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, c.device), "cudaDeviceGetAttribute");
    c.l2_bytes = v > 0 ? v : 1;
  }
  return bytes_per_voxel * g.nx * g.ny * g.nz <= (double)c.l2_bytes;
}

Grid grid_of(const fir_ctx& c, const VolInfo& v)
{
  const double vox[3] = {v.d.voxel_x, v.d.voxel_y, v.d.voxel_z};
  Grid g;
  g.nx = v.d.nx;
  g.ny = v.d.ny;
  g.nz = v.d.nz;
  g.nxy = v.d.nx * v.d.ny;
  for (int d = 0; d < 3; ++d)
  {
    if (c.geometry == FIR_GEOMETRY_REFERENCE)
    {
      // Siddon.h:113 keeps the voxel extents as int
      g.ext[d] = (double)(int)vox[d];
      if (g.ext[d] <= 0.0)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "voxel extent ", vox[d],
             " mm truncates to 0 in FIR's traversal (use FIR_GEOMETRY_EXACT)");
      }
    }
    else
    {
      g.ext[d] = vox[d];
    }
  }
  for (int d = 0; d < 3; ++d)
  {
    g.rext[d] = 1.0 / g.ext[d];  // IEEE division: RN(1 / ext)
  }
  const double depth = v.d.nz * v.d.voxel_z;
  g.low[0] = v.d.offset_x - v.d.voxel_x / 2;
  g.low[1] = v.d.offset_y - v.d.voxel_y / 2;
  g.low[2] = v.d.offset_z - depth / 2;
  g.high[0] = g.low[0] + v.d.nx * v.d.voxel_x;
  g.high[1] = g.low[1] + v.d.ny * v.d.voxel_y;
  g.high[2] = g.low[2] + depth;
  // Each traversal step consumes at least one plane crossing; a dimension
  // has at most span/step + 2 crossings in [alphaMin, alphaMax] (a cancelled
  // dimension two).  With FIR's truncated extents the step can be shorter
  // than the voxel, so the bound is counted in steps, not voxels.
  double bound = 8.0;
  for (int d = 0; d < 3; ++d)
  {
    bound += std::ceil((g.high[d] - g.low[d]) / g.ext[d]) + 2.0;
  }
  if (!(bound < 1.0e9))
  {
    fail(FIR_ERR_NOT_SUPPORTED, "volume spans ", bound, " traversal steps");
  }
  g.guard = (int)bound;
  g.exact_only = 0;
  if (c.step_limit > 0)
  {
    g.guard = std::min(g.guard, c.step_limit);
    g.exact_only = 1;
  }
  return g;
}

// Enumeration of the views v = offset + stride * j < n_views, segment by
// segment in FIR's order.  With stride = n_subsets dividing the number of
// views this is FIR's subset `offset` (LORCache.cc:49-51, 115-133), and the
// enumeration bases are the same for every offset.  A stride that does not
// divide the number of views (a subset's views shared unevenly between
// ranks) gives the first offsets one view more than the last.
Sino sino_of_views(const ProjInfo& p, int stride, int offset)
{
  Sino s;
  std::memset(&s, 0, sizeof(s));
  s.n_rings = p.d.n_rings;
  s.n_cpr = p.d.n_crystals_per_ring;
  s.span = p.d.segment_span;
  s.half_span = p.g.half_span;
  s.n_segments = p.d.n_segments;
  s.seg_offset = p.g.seg_offset;
  s.tang_offset = p.g.tang_offset;
  s.n_views = p.g.n_views;
  s.n_tang = p.g.n_tang_coords;
  s.n_subsets = stride;
  s.subset = offset;
  const long long views = offset < s.n_views ? (s.n_views - offset + stride - 1) / stride : 0;
  long long base = 0, ebase = 0;
  for (int k = 0; k < s.n_segments; ++k)
  {
    s.seg_base[k] = (int)base;
    s.enum_base[k] = (int)ebase;
    s.n_axial[k] = p.n_axial[k];
    base += (long long)p.n_axial[k] * s.n_views * s.n_tang;
    ebase += (long long)p.n_axial[k] * views * s.n_tang;
  }
  s.seg_base[s.n_segments] = (int)base;
  s.enum_base[s.n_segments] = (int)ebase;
  s.n_enum = (int)ebase;
  return s;
}

Sino sino_of(const ProjInfo& p, int n_subsets, int subset) { return sino_of_views(p, n_subsets, subset); }

// Page-locked host memory (cudaHostAlloc / cudaHostRegister), which the copy
// engines read asynchronously.
bool is_pinned_host(const void* p)
{
  if (p == nullptr)
  {
    return false;
  }
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
  {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

bool is_device_ptr(const void* p)
{
  if (p == nullptr)
  {
    return false;
  }
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
  {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Gives device views of caller buffers.  Device pointers pass through; host
// pointers are copied into context-owned device buffers (in), and copied
// back when finish() runs (out).  A call with any host pointer is
// synchronous: finish() waits for the stream and reports device checks.
class Stager
{
public:
  explicit Stager(fir_ctx& c): c_(c) {}

  template<typename T>
  const T* in(const T* p, long long n)
  {
    return static_cast<const T*>(stage(const_cast<T*>(p), n * (long long)sizeof(T), true, false));
  }

  template<typename T>
  T* out(T* p, long long n)
  {
    return static_cast<T*>(stage(p, n * (long long)sizeof(T), false, true));
  }

  template<typename T>
  T* inout(T* p, long long n)
  {
    return static_cast<T*>(stage(p, n * (long long)sizeof(T), true, true));
  }

  bool host() const { return any_host_; }

  void finish()
  {
    for (auto& b : back_)
    {
      cuda_ok(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, c_.stream), "cudaMemcpyAsync D2H");
    }
    if (any_host_)
    {
      cuda_ok(cudaStreamSynchronize(c_.stream), "cudaStreamSynchronize");
    }
  }

private:
  struct Back
  {
    void* host;
    void* dev;
    size_t bytes;
  };

  void* stage(void* p, long long bytes, bool copy_in, bool copy_out)
  {
    if (p == nullptr || is_device_ptr(p))
    {
      return p;
    }
    any_host_ = true;
    if (slot_ >= c_.staging.size())
    {
      c_.staging.resize(slot_ + 1);
    }
    void* d = c_.staging[slot_++].ensure((size_t)std::max<long long>(bytes, 16));
    if (copy_in)
    {
      cuda_ok(cudaMemcpyAsync(d, p, (size_t)bytes, cudaMemcpyHostToDevice, c_.stream), "cudaMemcpyAsync H2D");
    }
    if (copy_out)
    {
      back_.push_back(Back{p, d, (size_t)bytes});
    }
    return d;
  }

  fir_ctx& c_;
  size_t slot_ = 0;
  bool any_host_ = false;
  std::vector<Back> back_;
};

void read_checks(fir_ctx& c)
{
  cuda_ok(cudaMemcpyAsync(c.check_host, c.check.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream),
          "cudaMemcpyAsync check word");
  cuda_ok(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
  const int word = *c.check_host;
  if (word != 0)
  {
    cuda_ok(cudaMemsetAsync(c.check.p, 0, sizeof(int), c.stream), "cudaMemsetAsync");
    if (word & kCheckWalkGuard)
    {
      fail(FIR_ERR_DEVICE_CHECK, "a Siddon traversal exceeded its iteration bound (non-finite coordinates?)");
    }
    fail(FIR_ERR_DEVICE_CHECK, "device check word ", word);
  }
}

void finish(fir_ctx& c, Stager& st)
{
  st.finish();
  if (st.host())
  {
    read_checks(c);
  }
}

Taps gauss_taps(float fwhm, double vox, bool double_sigma)
{
  // operations.cc:32-75: half width (int(6 sigma / voxel) + 1) / 2, weights
  // exp(-k^2 voxel^2 / (2 sigma^2)).  sigma is float for x and y (divisor
  // 2.3548f) and double for z (divisor 2.3548).
  Taps t;
  std::memset(&t, 0, sizeof(t));
  if (double_sigma)
  {
    const double sigma = fwhm / 2.3548;
    t.half = (static_cast<int>(6.0 * sigma / vox) + 1) / 2;
    if (t.half > kMaxHalfTaps)
    {
      fail(FIR_ERR_NOT_SUPPORTED, "Gaussian filter half width ", t.half, " exceeds ", kMaxHalfTaps);
    }
    for (int k = -t.half; k <= t.half; ++k)
    {
      t.w[t.half + k] = (float)std::exp(-(k * k * vox * vox) / (2 * sigma * sigma));
    }
  }
  else
  {
    const float sigma = fwhm / 2.3548f;
    t.half = (static_cast<int>(6.0 * sigma / vox) + 1) / 2;
    if (t.half > kMaxHalfTaps)
    {
      fail(FIR_ERR_NOT_SUPPORTED, "Gaussian filter half width ", t.half, " exceeds ", kMaxHalfTaps);
    }
    for (int k = -t.half; k <= t.half; ++k)
    {
      t.w[t.half + k] = (float)std::exp(-(k * k * vox * vox) / (2 * sigma * sigma));
    }
  }
  return t;
}

// operations::convolve on device memory, all frames of vol.
void convolve_device(fir_ctx& c, const VolInfo& v, float* img, const float fwhm[3], float cut)
{
  if (!(fwhm[0] > 0.0 && fwhm[1] > 0.0 && fwhm[2] > 0.0))
  {
    return;
  }
  const Taps tx = gauss_taps(fwhm[0], v.d.voxel_x, false);
  const Taps ty = gauss_taps(fwhm[1], v.d.voxel_y, false);
  const Taps tz = gauss_taps(fwhm[2], v.d.voxel_z, true);
  const size_t bytes = (size_t)v.nvox * sizeof(float);
  float* t1 = static_cast<float*>(c.conv1.ensure(bytes));
  float* t2 = static_cast<float*>(c.conv2.ensure(bytes));
  float* cp = cut > 0.0f ? static_cast<float*>(c.conv_copy.ensure(bytes)) : nullptr;
  const LaunchCfg cfg = cfg_of(c);
  const float f = fwhm[0] > fwhm[1] ? fwhm[0] : fwhm[1];
  for (int fr = 0; fr < v.d.n_frames; ++fr)
  {
    float* x = img + (size_t)fr * v.nvox;
    if (cp != nullptr)
    {
      cuda_ok(cudaMemcpyAsync(cp, x, bytes, cudaMemcpyDeviceToDevice, c.stream), "cudaMemcpyAsync");
    }
    launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 0, tx, x, t1, cfg);
    launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 1, ty, t1, t2, cfg);
    launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 2, tz, t2, x, cfg);
    after_launch(c, 3);
    if (cp != nullptr)
    {
      launch_conv_restore(v.d.nx, v.d.ny, v.d.nz, v.d.voxel_x, v.d.voxel_y, cut, f, cp, x, cfg);
      after_launch(c);
    }
  }
}

void cut_device(fir_ctx& c, const VolInfo& v, float* img, float cut, int frames)
{
  if (!(cut > 0.0f))
  {
    return;
  }
  for (int fr = 0; fr < frames; ++fr)
  {
    launch_cut_circle(v.d.nx, v.d.ny, v.d.nz, v.d.voxel_x, v.d.voxel_y, cut, img + (size_t)fr * v.nvox,
                      cfg_of(c));
    after_launch(c);
  }
}

void check_osem_params(const fir_osem_params* prm, const ProjInfo& p)
{
  if (prm == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "OSEM parameters are NULL");
  }
  check_subsets(p, prm->n_subsets);
  if (prm->n_iterations < 0)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "number of iterations must not be negative");
  }
}

// Device-pointer body of one OSEM sub-iteration.
void osem_subiteration_device(fir_ctx& c, const ProjInfo& p, const Tables& t, const Grid& g,
                              const VolInfo& v, const float* sino, const float* mult, const float* bias, float* img,
                              const float* sens_frame, const fir_osem_params* prm, int subset,
                              int subiter)
{
  float* bp = static_cast<float*>(c.bp.ensure((size_t)v.nvox * sizeof(float)));
  cuda_ok(cudaMemsetAsync(bp, 0, (size_t)v.nvox * sizeof(float), c.stream), "cudaMemsetAsync");
  const Sino s = sino_of(p, prm->n_subsets, subset);
  const float* bp_t = ratio_backproject(c, g, s, t, img, sino, mult, bias, bp, v.nvox, true);
  if (bp_t != nullptr)
  {
    launch_em_update_oriented(g.nx, g.ny, g.nz, img, bp, bp_t, sens_frame, cfg_of(c));
  }
  else
  {
    launch_em_update(v.nvox, img, bp, sens_frame, cfg_of(c));
  }
  after_launch(c);
  const bool conv = prm->convolution_interval > 0 && prm->fwhm_xyz[0] > 0.0 && prm->fwhm_xyz[1] > 0.0 &&
                    prm->fwhm_xyz[2] > 0.0;
  if (conv && subiter % prm->convolution_interval == 0)
  {
    convolve_device(c, v, img, prm->fwhm_xyz, prm->cut_radius);
  }
  cut_device(c, v, img, prm->cut_radius, 1);
}

// One sub-iteration of the resolution-modelling OSEM: the Gaussian B of the
// parameters is part of the system model (projection of B x, B applied to
// the backprojection, sens_frame already blurred).
void osem_psf_subiteration_device(fir_ctx& c, const ProjInfo& p, const Tables& t, const Grid& g,
                                  const VolInfo& v, const float* sino, const float* mult, const float* bias, float* img,
                                  const float* sens_frame, const fir_osem_params* prm, int subset, int subiter)
{
  const size_t bytes = (size_t)v.nvox * sizeof(float);
  float* bp = static_cast<float*>(c.bp.ensure(bytes));
  float* blur = static_cast<float*>(c.psf_blur.ensure(bytes));
  cuda_ok(cudaMemsetAsync(bp, 0, bytes, c.stream), "cudaMemsetAsync");
  cuda_ok(cudaMemcpyAsync(blur, img, bytes, cudaMemcpyDeviceToDevice, c.stream), "cudaMemcpyAsync");
  convolve_device(c, v, blur, prm->fwhm_xyz, prm->cut_radius);
  const Sino s = sino_of(p, prm->n_subsets, subset);
  ratio_backproject(c, g, s, t, blur, sino, mult, bias, bp, v.nvox);
  convolve_device(c, v, bp, prm->fwhm_xyz, prm->cut_radius);
  launch_em_update(v.nvox, img, bp, sens_frame, cfg_of(c));
  after_launch(c);
  const bool conv = prm->convolution_interval > 0 && prm->fwhm_xyz[0] > 0.0 && prm->fwhm_xyz[1] > 0.0 &&
                    prm->fwhm_xyz[2] > 0.0;
  if (conv && subiter % prm->convolution_interval == 0)
  {
    convolve_device(c, v, img, prm->fwhm_xyz, prm->cut_radius);
  }
  cut_device(c, v, img, prm->cut_radius, 1);
}

// Input of an OSEM run copied subset by subset from pinned host memory, on a
// copy stream of the context, so that sub-iteration s of the first iteration
// waits only for its own bins and sensitivity frame: the copies of the next
// subsets overlap the computation.  Subset s holds views v with
// v % n_subsets == s (LORCache.cc:49-51), so in every segment its bins are
// view blocks at a fixed stride: one 2-D copy per segment and array.
class SubsetFeed
{
public:
  SubsetFeed(fir_ctx& c, const ProjInfo& p, long long nvox, int n_subsets): c_(c), p_(p), nvox_(nvox), nsub_(n_subsets)
  {
    if (c.copy_stream == nullptr)
    {
      cuda_ok(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    }
    while ((int)c.pipe_events.size() < n_subsets + 1)
    {
      cudaEvent_t e;
      cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
      c.pipe_events.push_back(e);
    }
    if (c.pipe.size() < 4)
    {
      c.pipe.resize(4);
    }
    // the previous call's kernels may still read the buffers
    cuda_ok(cudaEventRecord(c.pipe_events[n_subsets], c.stream), "cudaEventRecord");
    cuda_ok(cudaStreamWaitEvent(c.copy_stream, c.pipe_events[n_subsets], 0), "cudaStreamWaitEvent");
  }

  // Device buffer (slot 0..2) for a per-bin host array, or nullptr.
  const float* bins(int slot, const float* host)
  {
    if (host == nullptr)
    {
      return nullptr;
    }
    auto* d = static_cast<float*>(c_.pipe[(size_t)slot].ensure((size_t)p_.g.n_bins * sizeof(float)));
    arrays_.push_back({host, d});
    return d;
  }

  const float* frames(const float* host)
  {
    sens_host_ = host;
    sens_dev_ = static_cast<float*>(c_.pipe[3].ensure((size_t)nvox_ * nsub_ * sizeof(float)));
    return sens_dev_;
  }

  // Copies subset s and makes the context's stream wait for it.
  void feed(int s)
  {
    const int vps = p_.g.n_views / nsub_;
    size_t base = 0;
    for (int k = 0; k < p_.d.n_segments; ++k)
    {
      const size_t bpv = (size_t)p_.n_axial[(size_t)k] * p_.g.n_tang_coords;
      const size_t off = base + (size_t)s * bpv;
      const size_t pitch = (size_t)nsub_ * bpv * sizeof(float);
      for (const auto& a : arrays_)
      {
        cuda_ok(cudaMemcpy2DAsync(a.second + off, pitch, a.first + off, pitch, bpv * sizeof(float), (size_t)vps,
                                  cudaMemcpyHostToDevice, c_.copy_stream),
                "cudaMemcpy2DAsync");
      }
      base += bpv * (size_t)p_.g.n_views;
    }
    cuda_ok(cudaMemcpyAsync(sens_dev_ + (size_t)s * nvox_, sens_host_ + (size_t)s * nvox_,
                            (size_t)nvox_ * sizeof(float), cudaMemcpyHostToDevice, c_.copy_stream),
            "cudaMemcpyAsync");
    cuda_ok(cudaEventRecord(c_.pipe_events[(size_t)s], c_.copy_stream), "cudaEventRecord");
    cuda_ok(cudaStreamWaitEvent(c_.stream, c_.pipe_events[(size_t)s], 0), "cudaStreamWaitEvent");
  }

private:
  fir_ctx& c_;
  const ProjInfo& p_;
  long long nvox_;
  int nsub_;
  std::vector<std::pair<const float*, float*>> arrays_;
  const float* sens_host_ = nullptr;
  float* sens_dev_ = nullptr;
};

// The OSEM driver of fir_osem and fir_osem_psf (psf: resolution modelling).
void osem_run(fir_ctx& c, const fir_proj_desc* proj, const float* sino, const float* mult, const float* bias,
              const fir_vol_desc* vol,
              float* img, const float* sens, const fir_osem_params* params, fir_osem_save_fn save, void* user,
              bool psf)
{
  const ProjInfo p = check_proj(proj);
  check_osem_params(params, p);
  const VolInfo v = check_vol(vol);
  check_frames(v, 1);
  const Tables t = tables_of(c, p);
  const Grid g = grid_of(c, v);
  if (sino == nullptr || sens == nullptr || img == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "sinogram, image and sensitivity must not be NULL");
  }
  // pinned host inputs stream in subset by subset (the blurred sensitivity
  // of the PSF model needs all frames at once, so it is staged whole)
  const bool pipelined = !psf && is_pinned_host(sino) && is_pinned_host(sens) &&
                         (mult == nullptr || is_pinned_host(mult)) && (bias == nullptr || is_pinned_host(bias));
  Stager st(c);
  std::unique_ptr<SubsetFeed> feed;
  const float *dsino, *dmult, *dbias, *dsens;
  if (pipelined)
  {
    feed = std::make_unique<SubsetFeed>(c, p, v.nvox, params->n_subsets);
    dsino = feed->bins(0, sino);
    dmult = feed->bins(1, mult);
    dbias = feed->bins(2, bias);
    dsens = feed->frames(sens);
  }
  else
  {
    dsino = st.in(sino, p.g.n_bins);
    dmult = st.in(mult, p.g.n_bins);
    dbias = st.in(bias, p.g.n_bins);
    dsens = st.in(sens, v.nvox * params->n_subsets);
  }
  float* dimg = st.inout(img, v.nvox);
  if (psf)
  {
    // every subset's sensitivity frame blurred once: B A_s^T 1
    const size_t sbytes = (size_t)v.nvox * params->n_subsets * sizeof(float);
    float* sb = static_cast<float*>(c.psf_sens.ensure(sbytes));
    cuda_ok(cudaMemcpyAsync(sb, dsens, sbytes, cudaMemcpyDeviceToDevice, c.stream), "cudaMemcpyAsync");
    VolInfo frames = v;
    frames.d.n_frames = params->n_subsets;
    convolve_device(c, frames, sb, params->fwhm_xyz, params->cut_radius);
    dsens = sb;
  }
  std::vector<float> host_copy;
  cut_device(c, v, dimg, params->cut_radius, 1);
  const int nsub_total = params->n_iterations * params->n_subsets;
  for (int iter = 0; iter < params->n_iterations; ++iter)
  {
    for (int subset = 0; subset < params->n_subsets; ++subset)
    {
      const int subiter = iter * params->n_subsets + subset + 1;
      const float* sframe = dsens + (size_t)subset * v.nvox;
      if (feed && iter == 0)
      {
        feed->feed(subset);
      }
      if (psf)
      {
        osem_psf_subiteration_device(c, p, t, g, v, dsino, dmult, dbias, dimg, sframe, params, subset, subiter);
      }
      else
      {
        osem_subiteration_device(c, p, t, g, v, dsino, dmult, dbias, dimg, sframe, params, subset, subiter);
      }
      if (save != nullptr && params->save_interval > 0 && subiter % params->save_interval == 0 &&
          subiter != nsub_total)
      {
        host_copy.resize((size_t)v.nvox);
        cuda_ok(cudaMemcpyAsync(host_copy.data(), dimg, (size_t)v.nvox * sizeof(float), cudaMemcpyDeviceToHost,
                                c.stream),
                "cudaMemcpyAsync");
        cuda_ok(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
        save(user, subiter, host_copy.data());
      }
    }
  }
  finish(c, st);
}

// reconAlgos::OSEM_ResoReco as FIR runs it (reconAlgos.cc:203-367), with
// every image on the device for the whole run.  Its order of operations:
// the initial cut; every frame of the sensitivity volume filtered once, in
// place (operations::convolve filters all frames, operations.cc:77-187;
// reconAlgos.cc:232-236); then per sub-iteration the ratio backprojection of
// the unfiltered image (:270-312), the filtered backprojection,
// img <- img / sens_subset and img <- img * bp with the 1e-5 gates
// (:315-326), the post-filter every convolution_interval sub-iterations and
// the cut (:333-347).  FIR also filters a copy of the image every
// sub-iteration (`blur`, :264-268 and :350-353) but never reads it; that work
// has no effect and is not done.
void osem_reso_reco_run(fir_ctx& c, const fir_proj_desc* proj, const float* sino, const float* bias,
                        const fir_vol_desc* vol, float* img, float* sens, int n_sens_frames,
                        const fir_osem_params* params, fir_osem_save_fn save, void* user)
{
  const ProjInfo p = check_proj(proj);
  check_osem_params(params, p);
  const VolInfo v = check_vol(vol);
  check_frames(v, 1);
  if (n_sens_frames < params->n_subsets)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "Invalid frame");
  }
  const Tables t = tables_of(c, p);
  const Grid g = grid_of(c, v);
  if (sino == nullptr || sens == nullptr || img == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "sinogram, image and sensitivity must not be NULL");
  }
  Stager st(c);
  const float* dsino = st.in(sino, p.g.n_bins);
  const float* dbias = st.in(bias, p.g.n_bins);
  float* dsens = st.inout(sens, v.nvox * n_sens_frames);
  float* dimg = st.inout(img, v.nvox);
  const size_t bytes = (size_t)v.nvox * sizeof(float);
  float* bp = static_cast<float*>(c.bp.ensure(bytes));
  cut_device(c, v, dimg, params->cut_radius, 1);
  VolInfo frames = v;
  frames.d.n_frames = n_sens_frames;
  convolve_device(c, frames, dsens, params->fwhm_xyz, params->cut_radius);
  const bool conv = params->convolution_interval > 0 && params->fwhm_xyz[0] > 0.0 &&
                    params->fwhm_xyz[1] > 0.0 && params->fwhm_xyz[2] > 0.0;
  const int nsub_total = params->n_iterations * params->n_subsets;
  std::vector<float> host_copy;
  for (int iter = 0; iter < params->n_iterations; ++iter)
  {
    for (int subset = 0; subset < params->n_subsets; ++subset)
    {
      const int subiter = iter * params->n_subsets + subset + 1;
      cuda_ok(cudaMemsetAsync(bp, 0, bytes, c.stream), "cudaMemsetAsync");
      const Sino s = sino_of(p, params->n_subsets, subset);
      ratio_backproject(c, g, s, t, dimg, dsino, nullptr, dbias, bp, v.nvox);
      convolve_device(c, v, bp, params->fwhm_xyz, params->cut_radius);
      launch_em_update_image_first(v.nvox, dimg, bp, dsens + (size_t)subset * v.nvox, cfg_of(c));
      after_launch(c);
      if (conv && subiter % params->convolution_interval == 0)
      {
        convolve_device(c, v, dimg, params->fwhm_xyz, params->cut_radius);
      }
      cut_device(c, v, dimg, params->cut_radius, 1);
      if (save != nullptr && params->save_interval > 0 && subiter % params->save_interval == 0 &&
          subiter != nsub_total)
      {
        host_copy.resize((size_t)v.nvox);
        cuda_ok(cudaMemcpyAsync(host_copy.data(), dimg, bytes, cudaMemcpyDeviceToHost, c.stream), "cudaMemcpyAsync");
        cuda_ok(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
        save(user, subiter, host_copy.data());
      }
    }
  }
  finish(c, st);
}

}  // namespace fir::abi

using namespace fir;
using namespace fir::abi;

// ================================================================== ABI

extern "C" {

int fir_abi_version(void) { return FIR_CUDA_ABI_VERSION; }

const char* fir_last_error(void) { return g_error.c_str(); }

const char* fir_status_string(fir_status s)
{
  switch (s)
  {
  case FIR_OK: return "FIR_OK";
  case FIR_ERR_INVALID_ARGUMENT: return "FIR_ERR_INVALID_ARGUMENT";
  case FIR_ERR_CUDA: return "FIR_ERR_CUDA";
  case FIR_ERR_OUT_OF_MEMORY: return "FIR_ERR_OUT_OF_MEMORY";
  case FIR_ERR_DEVICE_CHECK: return "FIR_ERR_DEVICE_CHECK";
  case FIR_ERR_NO_DEVICE: return "FIR_ERR_NO_DEVICE";
  case FIR_ERR_NOT_SUPPORTED: return "FIR_ERR_NOT_SUPPORTED";
  }
  return "unknown fir_status";
}

fir_status fir_proj_geometry(const fir_proj_desc* desc, fir_proj_info* geom, int* n_axial)
{
  return guarded(__func__, [&] {
    const ProjInfo p = check_proj(desc);
    if (geom != nullptr)
    {
      *geom = p.g;
    }
    if (n_axial != nullptr)
    {
      std::copy(p.n_axial.begin(), p.n_axial.end(), n_axial);
    }
  });
}

fir_status fir_scanner_tables(const fir_scanner_desc* desc, double* xy, double* z, int* n_rings,
                              int* n_crystals_per_ring)
{
  return guarded(__func__, [&] {
    const ScannerInfo s = scanner_tables(desc, xy != nullptr || z != nullptr);
    if (n_rings != nullptr)
    {
      *n_rings = s.n_rings;
    }
    if (n_crystals_per_ring != nullptr)
    {
      *n_crystals_per_ring = s.n_cpr;
    }
    if (xy != nullptr)
    {
      std::copy(s.xy.begin(), s.xy.end(), xy);
    }
    if (z != nullptr)
    {
      std::copy(s.z.begin(), s.z.end(), z);
    }
  });
}

fir_status fir_ctx_create(fir_ctx** out, int device)
{
  return guarded(__func__, [&] {
    if (out == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "output pointer is NULL");
    }
    *out = nullptr;
    int n = 0;
    cuda_ok(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (device < 0 || device >= n)
    {
      fail(FIR_ERR_NO_DEVICE, "device ", device, " not present (", n, " visible)");
    }
    cuda_ok(cudaSetDevice(device), "cudaSetDevice");
    auto* c = new fir_ctx();
    c->device = device;
    try
    {
      c->check.ensure(sizeof(int));
      cuda_ok(cudaMemset(c->check.p, 0, sizeof(int)), "cudaMemset");
      cuda_ok(cudaMallocHost(&c->check_host, sizeof(int)), "cudaMallocHost");
    }
    catch (...)
    {
      c->check.release();
      delete c;
      throw;
    }
    *out = c;
  });
}

fir_status fir_ctx_destroy(fir_ctx* c)
{
  return guarded(__func__, [&] {
    if (c == nullptr)
    {
      return;
    }
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (DevBuf* b : {&c->xy, &c->z, &c->check, &c->bp, &c->conv1, &c->conv2, &c->conv_copy, &c->mu, &c->wide,
                      &c->det, &c->det_pairs, &c->ratio, &c->frames_il, &c->frames_acc, &c->psf_blur, &c->psf_sens, &c->rebin,
                      &c->wide_t, &c->bp_t, &c->img_t, &c->frames_il_t, &c->frames_acc_t, &c->compact})
    {
      b->release();
    }
    for (auto& b : c->staging)
    {
      b.release();
    }
    if (c->copy_stream != nullptr)
    {
      cudaStreamSynchronize(c->copy_stream);
      cudaStreamDestroy(c->copy_stream);
    }
    for (auto& b : c->pipe)
    {
      b.release();
    }
    for (auto e : c->pipe_events)
    {
      cudaEventDestroy(e);
    }
    for (auto& p : c->ev_pending)
    {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
    for (auto e : c->ev_pool)
    {
      cudaEventDestroy(e);
    }
    if (c->check_host != nullptr)
    {
      cudaFreeHost(c->check_host);
    }
    delete c;
  });
}

fir_status fir_ctx_set_stream(fir_ctx* ctx, void* stream)
{
  return guarded(__func__, [&] { check_ctx(ctx).stream = static_cast<cudaStream_t>(stream); });
}

fir_status fir_ctx_set_option(fir_ctx* ctx, fir_option opt, int value)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    switch (opt)
    {
    case FIR_OPT_GEOMETRY:
      if (value != FIR_GEOMETRY_REFERENCE && value != FIR_GEOMETRY_EXACT)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "unknown geometry mode ", value);
      }
      c.geometry = value;
      break;
    case FIR_OPT_BACKPROJ_MODE:
      if (value != FIR_BACKPROJ_ATOMIC && value != FIR_BACKPROJ_DETERMINISTIC)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "unknown backprojection mode ", value);
      }
      c.backproj = value;
      break;
    case FIR_OPT_SKIP_ZERO_BINS:
      c.skip_zero = value != 0;
      break;
    case FIR_OPT_BLOCK_SIZE:
      if (value == 0)
      {
        value = 128;
      }
      if (value < 32 || value > 256 || value % 32 != 0)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "block size must be a multiple of 32 in [32, 256]");
      }
      c.block = value;
      break;
    case FIR_OPT_TIMING:
      c.timing = value != 0;
      break;
    case FIR_OPT_STEP_LIMIT:
      if (value < 0)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "step limit must not be negative");
      }
      c.step_limit = value;
      break;
    case FIR_OPT_TRAVERSAL:
      if (value != FIR_TRAVERSAL_EXACT && value != FIR_TRAVERSAL_FLOAT)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "unknown traversal mode ", value);
      }
      c.traversal = value;
      break;
    case FIR_OPT_DETERMINISTIC_CHUNK:
      if (value < 0)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "chunk size must not be negative");
      }
      // at most 2^30 pairs per chunk (32 GiB of buffers), the sort's item limit
      c.det_chunk = value == 0 ? (1LL << 28) : std::min<long long>(value, 1LL << 30);
      break;
    default:
      fail(FIR_ERR_INVALID_ARGUMENT, "unknown option ", (int)opt);
    }
  });
}

fir_status fir_ctx_projector_time(fir_ctx* ctx, double* ms, long long* launches, int reset)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    drain_timing(c);
    if (ms != nullptr)
    {
      *ms = c.timed_ms;
    }
    if (launches != nullptr)
    {
      *launches = c.timed_n;
    }
    if (reset)
    {
      c.timed_ms = 0.0;
      c.timed_n = 0;
    }
  });
}

fir_status fir_ctx_get_option(fir_ctx* ctx, fir_option opt, int* value)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    if (value == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "output pointer is NULL");
    }
    switch (opt)
    {
    case FIR_OPT_GEOMETRY: *value = c.geometry; break;
    case FIR_OPT_BACKPROJ_MODE: *value = c.backproj; break;
    case FIR_OPT_SKIP_ZERO_BINS: *value = c.skip_zero; break;
    case FIR_OPT_BLOCK_SIZE: *value = c.block; break;
    case FIR_OPT_TIMING: *value = c.timing ? 1 : 0; break;
    case FIR_OPT_DETERMINISTIC_CHUNK: *value = (int)std::min<long long>(c.det_chunk, 0x7fffffff); break;
    case FIR_OPT_STEP_LIMIT: *value = c.step_limit; break;
    case FIR_OPT_TRAVERSAL: *value = c.traversal; break;
    default: fail(FIR_ERR_INVALID_ARGUMENT, "unknown option ", (int)opt);
    }
  });
}

fir_status fir_ctx_set_scanner(fir_ctx* ctx, const fir_scanner_desc* scanner)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ScannerInfo s = scanner_tables(scanner, true);
    cuda_ok(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
    c.xy.ensure(s.xy.size() * sizeof(double));
    c.z.ensure(s.z.size() * sizeof(double));
    cuda_ok(cudaMemcpy(c.xy.p, s.xy.data(), s.xy.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    cuda_ok(cudaMemcpy(c.z.p, s.z.data(), s.z.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    c.scan_rings = s.n_rings;
    c.scan_cpr = s.n_cpr;
    c.have_scanner = true;
  });
}

fir_status fir_ctx_synchronize(fir_ctx* ctx)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    read_checks(c);
  });
}

long long fir_ctx_launch_count(const fir_ctx* ctx) { return ctx != nullptr ? ctx->launches : -1; }

fir_status fir_forward(fir_ctx* ctx, const fir_vol_desc* vol, const float* img, const fir_proj_desc* proj,
                       float* sino)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    const ProjInfo p = check_proj(proj);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    Stager st(c);
    const float* dimg = st.in(img, v.nvox);
    float* dsino = st.out(sino, p.g.n_bins);
    const Sino s = sino_of(p, 1, 0);
    const Widened w = widen_for_projection(c, g, dimg);
    timed_launch(c, [&] { launch_forward(g, s, t, w.img, w.img_t, dsino, FwdEpilogue::None, cfg_of(c)); });
    finish(c, st);
  });
}

fir_status fir_forward_exp(fir_ctx* ctx, const fir_vol_desc* vol, const float* mu, const fir_proj_desc* proj,
                           float* acf)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    const ProjInfo p = check_proj(proj);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    Stager st(c);
    const float* dmu = st.in(mu, v.nvox);
    float* dacf = st.out(acf, p.g.n_bins);
    const Sino s = sino_of(p, 1, 0);
    const Widened w = widen_for_projection(c, g, dmu);
    timed_launch(c, [&] { launch_forward(g, s, t, w.img, w.img_t, dacf, FwdEpilogue::Exp, cfg_of(c)); });
    finish(c, st);
  });
}

fir_status fir_backward(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const fir_vol_desc* vol,
                        float* img, int n_subsets)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    check_subsets(p, n_subsets);
    const VolInfo v = check_vol(vol);
    check_frames(v, n_subsets);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (sino == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram is NULL");
    }
    Stager st(c);
    const float* dsino = st.in(sino, p.g.n_bins);
    float* dimg = st.out(img, v.nvox * n_subsets);
    cuda_ok(cudaMemsetAsync(dimg, 0, (size_t)(v.nvox * n_subsets) * sizeof(float), c.stream), "cudaMemsetAsync");
    for (int s = 0; s < n_subsets; ++s)
    {
      const Sino ss = sino_of(p, n_subsets, s);
      if (c.backproj == FIR_BACKPROJ_DETERMINISTIC)
      {
        det_backproject(c, g, ss, t, dsino, false, dimg + (size_t)s * v.nvox, v.nvox);
        continue;
      }
      backproject_subset(c, g, ss, t, dsino, dimg + (size_t)s * v.nvox, c.skip_zero != 0);
    }
    finish(c, st);
  });
}

static bool check_dtype(fir_dtype d)
{
  if (d != FIR_F32 && d != FIR_F64)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "unknown data type ", (int)d);
  }
  return d == FIR_F64;
}

fir_status fir_forward_frames(fir_ctx* ctx, const fir_vol_desc* vol, const void* img, const fir_proj_desc* proj,
                              void* sino, fir_dtype dtype)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    const ProjInfo p = check_proj(proj);
    const bool f64 = check_dtype(dtype);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (img == nullptr || sino == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "image and sinogram must not be NULL");
    }
    const long long es = f64 ? 8 : 4;
    const int nfr = v.d.n_frames;
    Stager st(c);
    const char* dimg = st.in(static_cast<const char*>(img), v.nvox * nfr * es);
    char* dsino = st.out(static_cast<char*>(sino), p.g.n_bins * nfr * es);
    const Sino s = sino_of(p, 1, 0);
    for (int f0 = 0; f0 < nfr; f0 += kMaxFramesPerPass)
    {
      const int nf = std::min(kMaxFramesPerPass, nfr - f0);
      const size_t il_bytes = (size_t)v.nvox * frames_stride(nf) * sizeof(double);
      auto* il = static_cast<double*>(c.frames_il.ensure(il_bytes));
      auto* il_t = use_exchanged(c, g, 2.0 * frames_stride(nf) * sizeof(double))
                       ? static_cast<double*>(c.frames_il_t.ensure(il_bytes))
                       : nullptr;
      launch_interleave(v.nvox, nf, g.nx, g.ny, dimg + (size_t)f0 * v.nvox * es, f64, il, il_t, cfg_of(c));
      after_launch(c);
      timed_launch(c, [&] {
        launch_forward_frames(g, s, t, il, il_t, nf, p.g.n_bins, dsino + (size_t)f0 * p.g.n_bins * es, f64,
                              cfg_of(c));
      });
    }
    finish(c, st);
  });
}

fir_status fir_backward_frames(fir_ctx* ctx, const fir_proj_desc* proj, const void* sino, const fir_vol_desc* vol,
                               void* img, fir_dtype dtype)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    const VolInfo v = check_vol(vol);
    const bool f64 = check_dtype(dtype);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (img == nullptr || sino == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "image and sinogram must not be NULL");
    }
    const long long es = f64 ? 8 : 4;
    const int nfr = v.d.n_frames;
    Stager st(c);
    const char* dsino = st.in(static_cast<const char*>(sino), p.g.n_bins * nfr * es);
    char* dimg = st.out(static_cast<char*>(img), v.nvox * nfr * es);
    const Sino s = sino_of(p, 1, 0);
    for (int f0 = 0; f0 < nfr; f0 += kMaxFramesPerPass)
    {
      const int nf = std::min(kMaxFramesPerPass, nfr - f0);
      const size_t acc_bytes = (size_t)v.nvox * frames_stride(nf) * es;
      void* acc = c.frames_acc.ensure(acc_bytes);
      cuda_ok(cudaMemsetAsync(acc, 0, acc_bytes, c.stream), "cudaMemsetAsync");
      void* acc_t = nullptr;
      if (use_exchanged(c, g, 2.0 * frames_stride(nf) * es))
      {
        acc_t = c.frames_acc_t.ensure(acc_bytes);
        cuda_ok(cudaMemsetAsync(acc_t, 0, acc_bytes, c.stream), "cudaMemsetAsync");
      }
      timed_launch(c, [&] {
        launch_backward_frames(g, s, t, dsino + (size_t)f0 * p.g.n_bins * es, nf, p.g.n_bins, acc, acc_t, f64,
                               c.skip_zero != 0, cfg_of(c));
      });
      launch_deinterleave(v.nvox, nf, g.nx, g.ny, acc, acc_t, f64, dimg + (size_t)f0 * v.nvox * es, cfg_of(c));
      after_launch(c);
    }
    finish(c, st);
  });
}

fir_status fir_sensitivity(fir_ctx* ctx, const fir_proj_desc* proj, const fir_vol_desc* vol, float* sens,
                           int n_subsets)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    check_subsets(p, n_subsets);
    const VolInfo v = check_vol(vol);
    check_frames(v, n_subsets);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    Stager st(c);
    float* dsens = st.out(sens, v.nvox * n_subsets);
    cuda_ok(cudaMemsetAsync(dsens, 0, (size_t)(v.nvox * n_subsets) * sizeof(float), c.stream), "cudaMemsetAsync");
    for (int s = 0; s < n_subsets; ++s)
    {
      const Sino ss = sino_of(p, n_subsets, s);
      if (c.backproj == FIR_BACKPROJ_DETERMINISTIC)
      {
        det_backproject(c, g, ss, t, nullptr, false, dsens + (size_t)s * v.nvox, v.nvox);
        continue;
      }
      backproject_subset(c, g, ss, t, nullptr, dsens + (size_t)s * v.nvox, false);
    }
    finish(c, st);
  });
}

fir_status fir_osem_subiteration(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                                 const fir_vol_desc* vol, float* img, const float* sens_frame,
                                 const fir_osem_params* params, int subset, int subiter)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    check_osem_params(params, p);
    if (subset < 0 || subset >= params->n_subsets)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "subset ", subset, " out of range [0, ", params->n_subsets, ")");
    }
    const VolInfo v = check_vol(vol);
    check_frames(v, 1);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (sino == nullptr || sens_frame == nullptr || img == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram, image and sensitivity must not be NULL");
    }
    Stager st(c);
    const float* dsino = st.in(sino, p.g.n_bins);
    const float* dbias = st.in(bias, p.g.n_bins);
    const float* dsens = st.in(sens_frame, v.nvox);
    float* dimg = st.inout(img, v.nvox);
    osem_subiteration_device(c, p, t, g, v, dsino, nullptr, dbias, dimg, dsens, params, subset, subiter);
    finish(c, st);
  });
}

fir_status fir_osem(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                    const fir_vol_desc* vol, float* img, const float* sens, const fir_osem_params* params,
                    fir_osem_save_fn save, void* user)
{
  return guarded(__func__, [&] { osem_run(check_ctx(ctx), proj, sino, nullptr, bias, vol, img, sens, params, save, user, false);
  });
}

fir_status fir_osem_psf(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                        const fir_vol_desc* vol, float* img, const float* sens, const fir_osem_params* params,
                        fir_osem_save_fn save, void* user)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const bool psf = params != nullptr && params->fwhm_xyz[0] > 0.0f && params->fwhm_xyz[1] > 0.0f &&
                     params->fwhm_xyz[2] > 0.0f;
    osem_run(c, proj, sino, nullptr, bias, vol, img, sens, params, save, user, psf);
  });
}

fir_status fir_osem_reso_reco(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                              const fir_vol_desc* vol, float* img, float* sens, int n_sens_frames,
                              const fir_osem_params* params, fir_osem_save_fn save, void* user)
{
  return guarded(__func__, [&] {
    osem_reso_reco_run(check_ctx(ctx), proj, sino, bias, vol, img, sens, n_sens_frames, params, save, user);
  });
}

fir_status fir_osem_weighted(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* mult,
                             const float* bias, const fir_vol_desc* vol, float* img, const float* sens,
                             const fir_osem_params* params, fir_osem_save_fn save, void* user)
{
  return guarded(__func__, [&] {
    if (mult == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "multiplicative factors must not be NULL");
    }
    osem_run(check_ctx(ctx), proj, sino, mult, bias, vol, img, sens, params, save, user, false);
  });
}

fir_status fir_ratio_backprojection(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino, const float* bias,
                                    const fir_vol_desc* vol, const float* img, float* bp, int n_subsets, int subset)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    check_subsets(p, n_subsets);
    if (subset < 0 || subset >= n_subsets)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "subset ", subset, " out of range [0, ", n_subsets, ")");
    }
    const VolInfo v = check_vol(vol);
    check_frames(v, 1);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (sino == nullptr || img == nullptr || bp == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram, image and backprojection must not be NULL");
    }
    Stager st(c);
    const float* dsino = st.in(sino, p.g.n_bins);
    const float* dbias = st.in(bias, p.g.n_bins);
    const float* dimg = st.in(img, v.nvox);
    float* dbp = st.out(bp, v.nvox);
    cuda_ok(cudaMemsetAsync(dbp, 0, (size_t)v.nvox * sizeof(float), c.stream), "cudaMemsetAsync");
    const Sino s = sino_of(p, n_subsets, subset);
    ratio_backproject(c, g, s, t, dimg, dsino, nullptr, dbias, dbp, v.nvox);
    finish(c, st);
  });
}

fir_status fir_ratio_backprojection_shard(fir_ctx* ctx, const fir_proj_desc* proj, const float* sino,
                                          const float* bias, const fir_vol_desc* vol, const float* img, float* bp,
                                          int n_subsets, int subset, int n_shards, int shard)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    check_subsets(p, n_subsets);
    if (subset < 0 || subset >= n_subsets)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "subset ", subset, " out of range [0, ", n_subsets, ")");
    }
    if (n_shards <= 0 || shard < 0 || shard >= n_shards || (long long)n_subsets * n_shards > (1LL << 30))
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "shard ", shard, " of ", n_shards, " is not valid");
    }
    const VolInfo v = check_vol(vol);
    check_frames(v, 1);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (sino == nullptr || img == nullptr || bp == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram, image and backprojection must not be NULL");
    }
    Stager st(c);
    const float* dsino = st.in(sino, p.g.n_bins);
    const float* dbias = st.in(bias, p.g.n_bins);
    const float* dimg = st.in(img, v.nvox);
    float* dbp = st.out(bp, v.nvox);
    cuda_ok(cudaMemsetAsync(dbp, 0, (size_t)v.nvox * sizeof(float), c.stream), "cudaMemsetAsync");
    // the subset's views subset + n_subsets * k with k % n_shards == shard
    const Sino s = sino_of_views(p, n_subsets * n_shards, subset + n_subsets * shard);
    if (s.n_enum > 0)
    {
      ratio_backproject(c, g, s, t, dimg, dsino, nullptr, dbias, dbp, v.nvox);
    }
    finish(c, st);
  });
}

fir_status fir_em_update(fir_ctx* ctx, const fir_vol_desc* vol, float* img, float* bp, const float* sens_frame)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    Stager st(c);
    float* dimg = st.inout(img, v.nvox);
    float* dbp = st.inout(bp, v.nvox);
    const float* dsens = st.in(sens_frame, v.nvox);
    launch_em_update(v.nvox, dimg, dbp, dsens, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_convolve(fir_ctx* ctx, const fir_vol_desc* vol, float* img, const float fwhm_xyz[3],
                        float cut_radius)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    if (fwhm_xyz == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "fwhm is NULL");
    }
    Stager st(c);
    float* dimg = st.inout(img, v.nvox * v.d.n_frames);
    convolve_device(c, v, dimg, fwhm_xyz, cut_radius);
    finish(c, st);
  });
}

fir_status fir_cut_circle(fir_ctx* ctx, const fir_vol_desc* vol, float* img, float cut_radius)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    Stager st(c);
    float* dimg = st.inout(img, v.nvox);
    cut_device(c, v, dimg, cut_radius, 1);
    finish(c, st);
  });
}

fir_status fir_apply_mask(fir_ctx* ctx, const fir_vol_desc* vol, float* img, const float* mask)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    Stager st(c);
    float* dimg = st.inout(img, v.nvox);
    const float* dmask = st.in(mask, v.nvox);
    launch_apply_mask(v.nvox, dimg, dmask, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_hu_to_mu(fir_ctx* ctx, const fir_vol_desc* vol, float* img)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    Stager st(c);
    float* dimg = st.inout(img, v.nvox);
    launch_hu_to_mu(v.nvox, dimg, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_proj_exponential(fir_ctx* ctx, const fir_proj_desc* proj, float* sino)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    Stager st(c);
    float* d = st.inout(sino, p.g.n_bins);
    launch_exponential(p.g.n_bins, d, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_proj_multiply(fir_ctx* ctx, const fir_proj_desc* proj, float* a, const float* b)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    Stager st(c);
    float* da = st.inout(a, p.g.n_bins);
    const float* db = st.in(b, p.g.n_bins);
    launch_proj_multiply(p.g.n_bins, da, db, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

// The (segment, axial) factors of ProjData::rebinWeight (ProjData.cc:541-615),
// one float per row of a span > 1 sinogram, 1 where FIR leaves the row
// alone: the ring differences of one ring sum are walked from the most
// negative, grouped into the segments' bands, and a band that merges w > 1
// of them gets (float)(1.0 / w).  FIR writes these rows through
// ProjData::weightBin, whose index adds the segment offset twice
// (ProjData.inl:76-79 with ProjHeader.inl:55) and leaves the arrays once
// there is more than one segment; here each factor goes to the row the
// algorithm names.
static std::vector<float> rebin_factors(const ProjInfo& p, int max_axial)
{
  const int ns = p.d.n_segments, span = p.d.segment_span, nr = p.d.n_rings;
  const int seg_off = p.g.seg_offset, mrd = p.g.max_ring_diff;
  std::vector<float> t((size_t)ns * max_axial, 1.0f);
  std::vector<char> hit((size_t)ns * max_axial, 0);
  for (int rs = 0; rs <= 2 * (nr - 1); ++rs)
  {
    int lmd = std::min(rs <= nr - 1 ? rs : 2 * (nr - 1) - rs, mrd);
    if ((rs + lmd) % 2 != 0)
    {
      --lmd;
    }
    int seg = -seg_off - 1;
    int next = -mrd - 1;
    while (next < -lmd)
    {
      ++seg;
      next += span;
    }
    int w = 1;
    for (int rd = -lmd; rd <= lmd; rd += 2)
    {
      if (rd == lmd || rd + 1 >= next)
      {
        if (w > 1)
        {
          const int aseg = seg < 0 ? -seg : seg;
          const int ax = seg == 0 ? rs : rs - (span + 1) / 2 - (aseg - 1) * span;
          const int si = seg + seg_off;
          if (si < 0 || si >= ns || ax < 0 || ax >= p.n_axial[(size_t)si])
          {
            fail(FIR_ERR_NOT_SUPPORTED, "rebin weight row (segment ", seg, ", axial ", ax, ") outside the sinogram");
          }
          const size_t k = (size_t)si * max_axial + ax;
          if (hit[k])
          {
            fail(FIR_ERR_NOT_SUPPORTED, "rebin weight row (segment ", seg, ", axial ", ax, ") weighted twice");
          }
          hit[k] = 1;
          t[k] = (float)(1.0 / w);
        }
        w = 1;
        ++seg;
        next += span;
      }
      else
      {
        ++w;
      }
    }
  }
  return t;
}

fir_status fir_bin_coordinates(fir_ctx* ctx, const fir_proj_desc* proj, long long n, const int* pairs, int* coords,
                               long long* bins)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    if (n < 0 || (n > 0 && pairs == nullptr))
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "n must be >= 0 and pairs non-NULL");
    }
    if (n == 0)
    {
      return;
    }
    Stager st(c);
    const int* dpairs = st.in(pairs, 4 * n);
    int* dcoords = st.out(coords, 5 * n);
    long long* dbins = st.out(bins, n);
    if (reinterpret_cast<uintptr_t>(dpairs) % 16 != 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "device crystal pairs must be 16-byte aligned");
    }
    launch_bin_coordinates(sino_of(p, 1, 0), p.g.max_ring_diff, n, dpairs, dcoords, dbins, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_proj_rebin_weight(fir_ctx* ctx, const fir_proj_desc* proj, float* sino)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    if (sino == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram is NULL");
    }
    if (p.d.segment_span == 1)
    {
      return;  // ProjData.cc:543: nothing to do for span 1
    }
    const int max_axial = *std::max_element(p.n_axial.begin(), p.n_axial.end());
    const std::vector<float> table = rebin_factors(p, max_axial);
    Stager st(c);
    float* dsino = st.inout(sino, p.g.n_bins);
    float* dtable = static_cast<float*>(c.rebin.ensure(table.size() * sizeof(float)));
    cuda_ok(cudaMemcpyAsync(dtable, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice, c.stream),
            "cudaMemcpyAsync");
    launch_rebin_weight(sino_of(p, 1, 0), dtable, max_axial, dsino, cfg_of(c));
    after_launch(c);
    finish(c, st);
    // the table is pageable host memory: keep it until the copy is done
    cuda_ok(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
  });
}

fir_status fir_siddon_paths(fir_ctx* ctx, const fir_vol_desc* vol, long long n, const double* ends, int cap,
                            int* coords, double* lengths, int* counts, int* crosses)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const VolInfo v = check_vol(vol);
    const Grid g = grid_of(c, v);
    if (n < 0 || cap < 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "negative count");
    }
    Stager st(c);
    const double* de = st.in(ends, 6 * n);
    int* dco = st.out(coords, n * cap);
    double* dle = st.out(lengths, n * cap);
    int* dcn = st.out(counts, n);
    int* dcr = st.out(crosses, n);
    launch_siddon_paths(g, n, de, cap, dco, dle, dcn, dcr, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

fir_status fir_lor_paths(fir_ctx* ctx, const fir_proj_desc* proj, const fir_vol_desc* vol, long long n,
                         const long long* bins, int cap, int* coords, double* lengths, int* counts, int* crosses)
{
  return guarded(__func__, [&] {
    fir_ctx& c = check_ctx(ctx);
    const ProjInfo p = check_proj(proj);
    const VolInfo v = check_vol(vol);
    const Tables t = tables_of(c, p);
    const Grid g = grid_of(c, v);
    if (n < 0 || cap < 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "negative count");
    }
    Stager st(c);
    const long long* db = st.in(bins, n);
    int* dco = st.out(coords, n * cap);
    double* dle = st.out(lengths, n * cap);
    int* dcn = st.out(counts, n);
    int* dcr = st.out(crosses, n);
    launch_lor_paths(g, sino_of(p, 1, 0), t, n, db, cap, dco, dle, dcn, dcr, cfg_of(c));
    after_launch(c);
    finish(c, st);
  });
}

}  // extern "C"

// ====================================== OSEM sub-iteration without allocation
//
// fir_osem_subiteration_noalloc runs the same kernels as
// fir_osem_subiteration, but takes its scratch memory (backprojection
// accumulator, widened image, filter passes, pre-filter copy) from the
// file-scope array below instead of from a context, and touches no host
// memory, so it never allocates.  The array's device address is looked up
// once per device with cudaGetSymbolAddress; the name itself is only a host
// stand-in and is never passed to a kernel.  This file defines no kernel, so
// under CUDA's lazy module loading (the default) the array is reserved when
// that first lookup loads the module, not when the library is loaded.

namespace
{
constexpr long long kNoAllocMaxVoxels = 1LL << 20;
// per voxel: accumulator (float) + widened image (double) + two filter
// passes (float) + pre-filter copy (float)
constexpr size_t kNoAllocBytesPerVoxel = 4 + 8 + 4 + 4 + 4;
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxVoxels * kNoAllocBytesPerVoxel;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace
{
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set-up on the
// first call per device).
unsigned char* noalloc_scratch()
{
  int device = 0;
  cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
  if (device < 0 || device >= kNoAllocMaxDevices)
  {
    fail(FIR_ERR_NOT_SUPPORTED, "device ordinal ", device, " beyond ", kNoAllocMaxDevices);
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_address[device] == nullptr)
  {
    void* p = nullptr;
    cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    g_noalloc_address[device] = p;
  }
  return static_cast<unsigned char*>(g_noalloc_address[device]);
}

// p must be memory of the current device (where the scratch array and the
// kernels live) or managed memory.
void require_device(const void* p, const char* what, int device)
{
  if (p == nullptr)
  {
    return;
  }
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
  {
    cudaGetLastError();
    a.type = cudaMemoryTypeUnregistered;
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, what, " must be device memory for the no-allocation entry point");
  }
  if (a.type == cudaMemoryTypeDevice && a.device != device)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, what, " is memory of device ", a.device, ", the current device is ", device);
  }
}

// The stream must belong to the current device (NULL: its default stream).
void require_stream_on(cudaStream_t stream, int device)
{
  if (stream == nullptr)
  {
    return;
  }
  int d = -1;
  if (cudaStreamGetDevice(stream, &d) != cudaSuccess)
  {
    cudaGetLastError();
    fail(FIR_ERR_INVALID_ARGUMENT, "stream is not a valid CUDA stream");
  }
  if (d != device)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "stream belongs to device ", d, ", the current device is ", device);
  }
}
}  // namespace

extern "C" fir_status fir_osem_subiteration_noalloc(const fir_proj_desc* proj, const double* crystal_xy,
                                                    const double* slice_z, const float* sino, const float* bias,
                                                    const fir_vol_desc* vol, float* img, const float* sens_frame,
                                                    const fir_osem_params* params, int subset, int subiter,
                                                    int geometry, void* stream)
{
  return guarded(__func__, [&] {
    const ProjInfo p = check_proj(proj);
    check_osem_params(params, p);
    if (subset < 0 || subset >= params->n_subsets)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "subset ", subset, " out of range [0, ", params->n_subsets, ")");
    }
    const VolInfo v = check_vol(vol);
    check_frames(v, 1);
    if (v.nvox > kNoAllocMaxVoxels)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "volume of ", v.nvox, " voxels exceeds the no-allocation limit of ",
           kNoAllocMaxVoxels, " voxels");
    }
    if (geometry != FIR_GEOMETRY_REFERENCE && geometry != FIR_GEOMETRY_EXACT)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "unknown geometry mode ", geometry);
    }
    if (crystal_xy == nullptr || slice_z == nullptr || sino == nullptr || img == nullptr || sens_frame == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "tables, sinogram, image and sensitivity must not be NULL");
    }
    int device = 0;
    cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
    require_device(crystal_xy, "crystal_xy", device);
    require_device(slice_z, "slice_z", device);
    require_device(sino, "sino", device);
    require_device(bias, "bias", device);
    require_device(img, "img", device);
    require_device(sens_frame, "sens_frame", device);
    require_stream_on(static_cast<cudaStream_t>(stream), device);

    // geometry as a context in the requested mode would build it
    fir_ctx geo;
    geo.geometry = geometry;
    const Grid g = grid_of(geo, v);
    const Sino s = sino_of(p, params->n_subsets, subset);
    const Tables t{reinterpret_cast<const double2*>(crystal_xy), slice_z};

    unsigned char* base = noalloc_scratch();
    const size_t n = (size_t)kNoAllocMaxVoxels;
    float* bp = reinterpret_cast<float*>(base);
    double* wide = reinterpret_cast<double*>(base + 4 * n);
    float* t1 = reinterpret_cast<float*>(base + 12 * n);
    float* t2 = reinterpret_cast<float*>(base + 16 * n);
    float* copy = reinterpret_cast<float*>(base + 20 * n);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const LaunchCfg cfg{128, st, nullptr};

    // the accumulator keeps the previous call's sums: clear it
    cuda_ok(cudaMemsetAsync(bp, 0, (size_t)v.nvox * sizeof(float), st), "cudaMemsetAsync");
    launch_widen(v.nvox, img, wide, cfg);
    launch_osem_subset(g, s, t, wide, nullptr, sino, nullptr, bias, bp, nullptr, false, cfg);
    launch_em_update(v.nvox, img, bp, sens_frame, cfg);
    const float* fwhm = params->fwhm_xyz;
    const bool conv = params->convolution_interval > 0 && fwhm[0] > 0.0 && fwhm[1] > 0.0 && fwhm[2] > 0.0;
    if (conv && subiter % params->convolution_interval == 0)
    {
      const Taps tx = gauss_taps(fwhm[0], v.d.voxel_x, false);
      const Taps ty = gauss_taps(fwhm[1], v.d.voxel_y, false);
      const Taps tz = gauss_taps(fwhm[2], v.d.voxel_z, true);
      const float cut = params->cut_radius;
      if (cut > 0.0f)
      {
        cuda_ok(cudaMemcpyAsync(copy, img, (size_t)v.nvox * sizeof(float), cudaMemcpyDeviceToDevice, st),
                "cudaMemcpyAsync");
      }
      launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 0, tx, img, t1, cfg);
      launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 1, ty, t1, t2, cfg);
      launch_conv_pass(v.d.nx, v.d.ny, v.d.nz, 2, tz, t2, img, cfg);
      if (cut > 0.0f)
      {
        launch_conv_restore(v.d.nx, v.d.ny, v.d.nz, v.d.voxel_x, v.d.voxel_y, cut, fwhm[0] > fwhm[1] ? fwhm[0] : fwhm[1],
                            copy, img, cfg);
      }
    }
    if (params->cut_radius > 0.0f)
    {
      launch_cut_circle(v.d.nx, v.d.ny, v.d.nz, v.d.voxel_x, v.d.voxel_y, params->cut_radius, img, cfg);
    }
    cuda_ok(cudaGetLastError(), "kernel launch");
  });
}
