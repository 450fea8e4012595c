// C ABI of the batched OSEM (fir_batch_*, include/fir_cuda.h): many
// independent reconstructions run as one schedule.  Kernels in batch.cu.
#include "capi_common.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

using namespace fir;
using namespace fir::abi;

// ================================================================== batches
//
// fir_batch: many independent OSEM reconstructions run together (see
// batch.cu for the kernels).  The host builds, once, the per-problem device
// descriptors and the item lists of every step of the schedule:
//   prepare   all problems, voxel blocks          (initial cut, double copy)
//   step t    projector items (bundles of 32 LORs), EM items (voxel blocks),
//             filter items (voxel blocks of the problems that filter at t)
// Items of the projector are ordered by decreasing path length, so that the
// queue hands out the longest bundles first.
//
// A problem whose subsets alone fill the GPU many times over (kDirectLors),
// or whose volume fits L2 only as float image and accumulator, runs its
// projector as fir_osem does, in launches of its own within the step: the
// kernel then reads its descriptor from kernel parameters rather than from
// memory, which leaves the walk the registers it needs (the large 320x320x128
// problem: 358 ms of projector per iteration batched, 325 ms direct), and the
// float gathers run as one launch per orientation.

// 2^22 LORs per subset: 14 waves of 148 SMs x 2048 threads.
constexpr long long kDirectLors = 1LL << 22;

struct fir_batch
{
  struct Problem
  {
    ProjInfo p;
    VolInfo v;
    fir_osem_params prm;
    int n_subsets = 1;
    int n_sub_total = 0;
    int n_enum = 0;
    bool filter = false;
    bool exchanged = false;  // x/y-exchanged images for LORs along x (use_exchanged)
    bool gather_float = false;  // no double copy: too large for L2 beside the accumulator
    // the projector runs as fir_osem's kernel in launches of its own, its
    // descriptor as kernel parameters (kDirectLors)
    bool direct = false;
    double path = 0.0;  // nx + ny + nz: relative cost of a bundle
    size_t off_sino = 0, off_sens = 0, off_img = 0, off_wide = 0, off_bp = 0, off_wide_t = 0, off_bp_t = 0,
           off_img_t = 0, off_t1 = 0, off_t2 = 0, off_xy = 0, off_z = 0;
    DevBuf bias;
  };
  struct Launch
  {
    int item_off = 0, n_items = 0, n_units = 0;
  };
  struct Step
  {
    Launch proj, em, filt;
    std::vector<std::pair<int, int>> direct;  // (problem, subset) of the direct projector launches
  };

  fir_ctx* ctx = nullptr;
  int n = 0;
  int n_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<Problem> pr;
  std::vector<BatchProblem> desc_host;
  DevBuf arena, desc, items, queue;
  Launch all;
  std::vector<Step> steps;
  BatchLaunch shape{128, 0, 1};
  // the last fir_batch_tune: every candidate shape with its best time (ms)
  std::vector<std::pair<BatchLaunch, double>> tuned;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long schedule_launches = 0;
};

namespace
{
fir_batch& check_batch(fir_batch* b)
{
  if (b == nullptr)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "batch is NULL");
  }
  check_ctx(b->ctx);
  return *b;
}

fir_batch::Problem& batch_problem(fir_batch& b, int p)
{
  if (p < 0 || p >= b.n)
  {
    fail(FIR_ERR_INVALID_ARGUMENT, "problem index ", p, " out of range [0, ", b.n, ")");
  }
  return b.pr[(size_t)p];
}

void drop_graph(fir_batch& b)
{
  if (b.exec != nullptr)
  {
    cudaGraphExecDestroy(b.exec);
    b.exec = nullptr;
  }
  if (b.graph != nullptr)
  {
    cudaGraphDestroy(b.graph);
    b.graph = nullptr;
  }
}

void release_batch(fir_batch& b)
{
  drop_graph(b);
  for (auto& q : b.pr)
  {
    q.bias.release();
  }
  for (DevBuf* d : {&b.arena, &b.desc, &b.items, &b.queue})
  {
    d->release();
  }
  if (b.ev_in != nullptr)
  {
    cudaEventDestroy(b.ev_in);
  }
  if (b.ev_out != nullptr)
  {
    cudaEventDestroy(b.ev_out);
  }
  if (b.stream != nullptr)
  {
    cudaStreamDestroy(b.stream);
  }
}

// Appends a launch over the given problems (with per-problem subset and
// filter flag) to the item list; units per problem from `units`.
template<typename Units>
fir_batch::Launch add_launch(std::vector<BatchItem>& items, const std::vector<int>& problems,
                             const std::vector<int>& subsets, const std::vector<int>& filters, Units&& units)
{
  fir_batch::Launch L;
  L.item_off = (int)items.size();
  long long total = 0;
  for (size_t k = 0; k < problems.size(); ++k)
  {
    items.push_back(BatchItem{problems[k], subsets[k], filters[k], (int)total});
    total += units(problems[k]);
    if (total > 0x7fffffffLL)
    {
      fail(FIR_ERR_NOT_SUPPORTED, "batched launch of ", total, " work units exceeds 2^31-1");
    }
  }
  L.n_items = (int)problems.size();
  L.n_units = (int)total;
  return L;
}

void check_launch(cudaStream_t s)
{
  (void)s;
  cuda_ok(cudaGetLastError(), "kernel launch");
}

// Enqueues the batched projector launch of a step (queue: its zeroed counter).
void batch_project(fir_batch& b, const fir_batch::Launch& L, int* queue, const BatchLaunch& shape, cudaStream_t s)
{
  const auto* P = static_cast<const BatchProblem*>(b.desc.p);
  const auto* I = static_cast<const BatchItem*>(b.items.p) + L.item_off;
  launch_batch_project(P, I, L.n_items, L.n_units, queue, shape, b.n_sms, static_cast<int*>(b.ctx->check.p), s);
  check_launch(s);
}

// Enqueues problem k's projector for one subset as fir_osem runs it (one
// launch, two when it gathers floats); returns the number of launches.
long long direct_project(fir_batch& b, int k, int subset, cudaStream_t s)
{
  const BatchProblem& d = b.desc_host[(size_t)k];
  Sino sub = d.s;
  sub.subset = subset;
  const LaunchCfg cfg{b.ctx->block, s, static_cast<int*>(b.ctx->check.p)};
  if (b.pr[(size_t)k].gather_float)
  {
    launch_osem_subset_float_image(d.g, sub, d.t, d.img, d.img_t, d.sino, nullptr, d.bias, d.bp, d.bp_t,
                                   d.skip_zero != 0, cfg);
    check_launch(s);
    return d.img_t != nullptr ? 2 : 1;
  }
  launch_osem_subset(d.g, sub, d.t, d.wide, d.wide_t, d.sino, nullptr, d.bias, d.bp, d.bp_t, d.skip_zero != 0, cfg);
  check_launch(s);
  return 1;
}

// The whole schedule on stream s; returns the number of kernel launches.
long long batch_enqueue(fir_batch& b, cudaStream_t s)
{
  const auto* P = static_cast<const BatchProblem*>(b.desc.p);
  const auto* I = static_cast<const BatchItem*>(b.items.p);
  int* queue = static_cast<int*>(b.queue.p);
  long long n = 0;
  cuda_ok(cudaMemsetAsync(queue, 0, b.steps.size() * sizeof(int), s), "cudaMemsetAsync");
  launch_batch_prepare(P, I + b.all.item_off, b.all.n_items, b.all.n_units, true, s);
  check_launch(s);
  ++n;
  for (size_t t = 0; t < b.steps.size(); ++t)
  {
    const fir_batch::Step& st = b.steps[t];
    batch_project(b, st.proj, queue + t, b.shape, s);
    n += st.proj.n_items > 0 ? 1 : 0;
    for (const auto& ks : st.direct)
    {
      n += direct_project(b, ks.first, ks.second, s);
    }
    launch_batch_em(P, I + st.em.item_off, st.em.n_items, st.em.n_units, s);
    check_launch(s);
    ++n;
    if (st.filt.n_items > 0)
    {
      for (int axis = 0; axis < 3; ++axis)
      {
        launch_batch_filter(P, I + st.filt.item_off, st.filt.n_items, st.filt.n_units, axis, s);
        check_launch(s);
      }
      n += 3;
    }
  }
  return n;
}

void batch_copy(fir_batch& b, void* dst, const void* src, size_t bytes)
{
  cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, b.ctx->stream), "cudaMemcpyAsync");
}

// Builds the item lists of the whole schedule for the current launch shape
// (its bundle form sets the projector's work units) and uploads them with the
// problem descriptors; waits for the copies.
void build_schedule(fir_batch& b)
{
  const int n_problems = b.n;
  for (int k = 0; k < n_problems; ++k)
  {
    batch_bundle_bases(b.desc_host[(size_t)k].s, b.shape.axial_tile, b.desc_host[(size_t)k].bundle_base);
  }
  b.steps.clear();
  std::vector<BatchItem> items;
  std::vector<int> all((size_t)n_problems), zeros((size_t)n_problems, 0);
  for (int k = 0; k < n_problems; ++k)
  {
    all[(size_t)k] = k;
  }
  auto vox_units = [&](int k) { return (b.pr[(size_t)k].v.nvox + kBatchBlock - 1) / kBatchBlock; };
  auto lor_units = [&](int k) { return batch_bundles(b.desc_host[(size_t)k].s, b.shape.axial_tile); };
  b.all = add_launch(items, all, zeros, zeros, vox_units);
  std::vector<int> order = all;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b.pr[(size_t)x].path > b.pr[(size_t)y].path; });
  int n_steps = 0;
  for (const auto& q : b.pr)
  {
    n_steps = std::max(n_steps, q.n_sub_total);
  }
  for (int t = 0; t < n_steps; ++t)
  {
    std::vector<int> probs, subs, filts, fprobs, fsubs, fflags, dprobs, dsubs, dfilts;
    fir_batch::Step st;
    for (int k : order)
    {
      const fir_batch::Problem& q = b.pr[(size_t)k];
      if (t >= q.n_sub_total)
      {
        continue;
      }
      const int subiter = t + 1;
      const int f = q.filter && subiter % q.prm.convolution_interval == 0 ? 1 : 0;
      probs.push_back(k);
      subs.push_back(t % q.n_subsets);
      filts.push_back(f);
      if (q.direct)
      {
        st.direct.emplace_back(k, t % q.n_subsets);
      }
      else
      {
        dprobs.push_back(k);
        dsubs.push_back(t % q.n_subsets);
        dfilts.push_back(f);
      }
      if (f)
      {
        fprobs.push_back(k);
        fsubs.push_back(t % q.n_subsets);
        fflags.push_back(1);
      }
    }
    st.proj = add_launch(items, dprobs, dsubs, dfilts, lor_units);
    st.em = add_launch(items, probs, subs, filts, vox_units);
    st.filt = add_launch(items, fprobs, fsubs, fflags, vox_units);
    b.steps.push_back(st);
  }
  b.desc.ensure(b.desc_host.size() * sizeof(BatchProblem));
  batch_copy(b, b.desc.p, b.desc_host.data(), b.desc_host.size() * sizeof(BatchProblem));
  b.items.ensure(std::max<size_t>(items.size(), 1) * sizeof(BatchItem));
  batch_copy(b, b.items.p, items.data(), items.size() * sizeof(BatchItem));
  b.queue.ensure(std::max<size_t>(b.steps.size(), 1) * sizeof(int));
  cuda_ok(cudaStreamSynchronize(b.ctx->stream), "cudaStreamSynchronize");
  b.schedule_launches = 1;
  for (const auto& st : b.steps)
  {
    b.schedule_launches += 1 + (st.proj.n_items > 0 ? 1 : 0) + (st.filt.n_items > 0 ? 3 : 0);
    for (const auto& ks : st.direct)
    {
      const BatchProblem& d = b.desc_host[(size_t)ks.first];
      b.schedule_launches += d.img_t != nullptr ? 2 : 1;
    }
  }
}

// Makes s the launch shape: drops the captured graph, and rebuilds the
// schedule when the bundle form changes.
void set_shape(fir_batch& b, const BatchLaunch& s)
{
  const BatchLaunch& o = b.shape;
  if (s.block == o.block && s.blocks_per_sm == o.blocks_per_sm && s.grab == o.grab && s.axial_tile == o.axial_tile)
  {
    return;
  }
  cuda_ok(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
  drop_graph(b);
  const bool rebuild = s.axial_tile != o.axial_tile;
  b.shape = s;
  if (rebuild)
  {
    build_schedule(b);
  }
}

// Orders the batch's stream after the context's stream.
void batch_begin(fir_batch& b)
{
  cuda_ok(cudaEventRecord(b.ev_in, b.ctx->stream), "cudaEventRecord");
  cuda_ok(cudaStreamWaitEvent(b.stream, b.ev_in, 0), "cudaStreamWaitEvent");
}

// Orders the context's stream after the batch's stream.
void batch_end(fir_batch& b)
{
  cuda_ok(cudaEventRecord(b.ev_out, b.stream), "cudaEventRecord");
  cuda_ok(cudaStreamWaitEvent(b.ctx->stream, b.ev_out, 0), "cudaStreamWaitEvent");
}
}  // namespace

extern "C" {

fir_status fir_batch_create(fir_batch** out, fir_ctx* ctx, int n_problems, const fir_scanner_desc* scanners,
                            const fir_proj_desc* projs, const fir_vol_desc* vols, const fir_osem_params* params)
{
  return guarded(__func__, [&] {
    if (out == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "output pointer is NULL");
    }
    *out = nullptr;
    fir_ctx& c = check_ctx(ctx);
    if (n_problems <= 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "a batch needs at least one problem");
    }
    if (scanners == nullptr || projs == nullptr || vols == nullptr || params == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "scanner, projection, volume and parameter arrays must not be NULL");
    }
    auto b = std::make_unique<fir_batch>();
    b->ctx = ctx;
    b->n = n_problems;
    b->pr.resize((size_t)n_problems);
    std::vector<ScannerInfo> scan((size_t)n_problems);
    // validate and lay out the arena
    size_t off = 0;
    auto take = [&off](size_t bytes) {
      const size_t at = off;
      off += (bytes + 255) & ~(size_t)255;
      return at;
    };
    for (int k = 0; k < n_problems; ++k)
    {
      fir_batch::Problem& q = b->pr[(size_t)k];
      q.p = check_proj(&projs[k]);
      q.v = check_vol(&vols[k]);
      check_frames(q.v, 1);
      check_osem_params(&params[k], q.p);
      q.prm = params[k];
      scan[(size_t)k] = scanner_tables(&scanners[k], true);
      if (q.p.d.n_rings != scan[(size_t)k].n_rings || q.p.d.n_crystals_per_ring != scan[(size_t)k].n_cpr)
      {
        fail(FIR_ERR_INVALID_ARGUMENT, "problem ", k, ": Projection must have the same number of rings (",
             scan[(size_t)k].n_rings, ") and the same number of crystals per ring (", scan[(size_t)k].n_cpr,
             ") as the scanner");
      }
      q.n_subsets = q.prm.n_subsets;
      q.n_sub_total = q.prm.n_iterations * q.prm.n_subsets;
      q.filter = q.prm.convolution_interval > 0 && q.prm.fwhm_xyz[0] > 0.0f && q.prm.fwhm_xyz[1] > 0.0f &&
                 q.prm.fwhm_xyz[2] > 0.0f;
      q.path = (double)q.v.d.nx + q.v.d.ny + q.v.d.nz;
      const size_t nv = (size_t)q.v.nvox;
      q.off_sino = take((size_t)q.p.g.n_bins * sizeof(float));
      q.off_sens = take(nv * q.n_subsets * sizeof(float));
      q.off_img = take(nv * sizeof(float));
      {
        const Grid g = grid_of(c, q.v);
        q.exchanged = use_exchanged(c, g);
        q.gather_float = !q.exchanged && !use_exchanged(c, g, 12.0) && use_exchanged(c, g, 8.0);
      }
      q.off_wide = take(q.gather_float ? 0 : nv * sizeof(double));
      q.off_bp = take(nv * sizeof(float));
      q.off_wide_t = take(q.exchanged ? nv * sizeof(double) : 0);
      q.off_bp_t = take(q.exchanged || q.gather_float ? nv * sizeof(float) : 0);
      q.off_img_t = take(q.gather_float ? nv * sizeof(float) : 0);
      q.off_t1 = take(q.filter ? nv * sizeof(float) : 0);
      q.off_t2 = take(q.filter ? nv * sizeof(float) : 0);
      q.off_xy = take(scan[(size_t)k].xy.size() * sizeof(double));
      q.off_z = take(scan[(size_t)k].z.size() * sizeof(double));
    }
    b->desc_host.resize((size_t)n_problems);
    cuda_ok(cudaDeviceGetAttribute(&b->n_sms, cudaDevAttrMultiProcessorCount, c.device), "cudaDeviceGetAttribute");
    try
    {
      cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      cuda_ok(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming), "cudaEventCreate");
      cuda_ok(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming), "cudaEventCreate");
      auto* base = static_cast<unsigned char*>(b->arena.ensure(std::max<size_t>(off, 256)));
      cuda_ok(cudaMemsetAsync(base, 0, off, c.stream), "cudaMemsetAsync");
      for (int k = 0; k < n_problems; ++k)
      {
        fir_batch::Problem& q = b->pr[(size_t)k];
        BatchProblem& d = b->desc_host[(size_t)k];
        std::memset(&d, 0, sizeof(d));
        fir_ctx geo;
        geo.geometry = c.geometry;
        d.g = grid_of(geo, q.v);
        d.s = sino_of(q.p, q.n_subsets, 0);
        q.n_enum = d.s.n_enum;
        q.direct = q.gather_float || (long long)q.n_enum >= kDirectLors;
        batch_copy(*b, base + q.off_xy, scan[(size_t)k].xy.data(), scan[(size_t)k].xy.size() * sizeof(double));
        batch_copy(*b, base + q.off_z, scan[(size_t)k].z.data(), scan[(size_t)k].z.size() * sizeof(double));
        d.t = Tables{reinterpret_cast<const double2*>(base + q.off_xy), reinterpret_cast<const double*>(base + q.off_z)};
        d.sino = reinterpret_cast<const float*>(base + q.off_sino);
        d.bias = nullptr;
        d.sens = reinterpret_cast<const float*>(base + q.off_sens);
        d.img = reinterpret_cast<float*>(base + q.off_img);
        d.wide = q.gather_float ? nullptr : reinterpret_cast<double*>(base + q.off_wide);
        d.bp = reinterpret_cast<float*>(base + q.off_bp);
        d.wide_t = q.exchanged ? reinterpret_cast<double*>(base + q.off_wide_t) : nullptr;
        d.bp_t = q.exchanged || q.gather_float ? reinterpret_cast<float*>(base + q.off_bp_t) : nullptr;
        d.img_t = q.gather_float ? reinterpret_cast<float*>(base + q.off_img_t) : nullptr;
        d.t1 = q.filter ? reinterpret_cast<float*>(base + q.off_t1) : nullptr;
        d.t2 = q.filter ? reinterpret_cast<float*>(base + q.off_t2) : nullptr;
        d.nvox = (int)q.v.nvox;
        d.skip_zero = c.skip_zero;
        d.vx = q.v.d.voxel_x;
        d.vy = q.v.d.voxel_y;
        d.cut = q.prm.cut_radius > 0.0f ? q.prm.cut_radius : 0.0f;
        d.fwhm = q.prm.fwhm_xyz[0] > q.prm.fwhm_xyz[1] ? q.prm.fwhm_xyz[0] : q.prm.fwhm_xyz[1];
        if (q.filter)
        {
          d.tx = gauss_taps(q.prm.fwhm_xyz[0], q.v.d.voxel_x, false);
          d.ty = gauss_taps(q.prm.fwhm_xyz[1], q.v.d.voxel_y, false);
          d.tz = gauss_taps(q.prm.fwhm_xyz[2], q.v.d.voxel_z, true);
        }
      }
      build_schedule(*b);
    }
    catch (...)
    {
      release_batch(*b);
      throw;
    }
    *out = b.release();
  });
}

fir_status fir_batch_destroy(fir_batch* batch)
{
  return guarded(__func__, [&] {
    if (batch == nullptr)
    {
      return;
    }
    if (batch->ctx != nullptr)
    {
      cudaSetDevice(batch->ctx->device);
    }
    if (batch->stream != nullptr)
    {
      cudaStreamSynchronize(batch->stream);
    }
    release_batch(*batch);
    delete batch;
  });
}

fir_status fir_batch_set_data(fir_batch* batch, int p, const float* sino, const float* sens, const float* bias)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    fir_batch::Problem& q = batch_problem(b, p);
    if (sino == nullptr || sens == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "sinogram and sensitivity must not be NULL");
    }
    auto* base = static_cast<unsigned char*>(b.arena.p);
    cuda_ok(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
    batch_copy(b, base + q.off_sino, sino, (size_t)q.p.g.n_bins * sizeof(float));
    batch_copy(b, base + q.off_sens, sens, (size_t)q.v.nvox * q.n_subsets * sizeof(float));
    BatchProblem& d = b.desc_host[(size_t)p];
    const float* want = nullptr;
    if (bias != nullptr)
    {
      want = static_cast<const float*>(q.bias.ensure((size_t)q.p.g.n_bins * sizeof(float)));
      batch_copy(b, q.bias.p, bias, (size_t)q.p.g.n_bins * sizeof(float));
    }
    if (d.bias != want)
    {
      d.bias = want;
      batch_copy(b, static_cast<BatchProblem*>(b.desc.p) + p, &d, sizeof(BatchProblem));
      // a direct projector launch holds the bias pointer in its parameters
      drop_graph(b);
    }
    cuda_ok(cudaStreamSynchronize(b.ctx->stream), "cudaStreamSynchronize");
  });
}

fir_status fir_batch_set_image(fir_batch* batch, int p, const float* img)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    fir_batch::Problem& q = batch_problem(b, p);
    if (img == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "image must not be NULL");
    }
    cuda_ok(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
    batch_copy(b, static_cast<unsigned char*>(b.arena.p) + q.off_img, img, (size_t)q.v.nvox * sizeof(float));
    cuda_ok(cudaStreamSynchronize(b.ctx->stream), "cudaStreamSynchronize");
  });
}

fir_status fir_batch_get_image(fir_batch* batch, int p, float* img)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    fir_batch::Problem& q = batch_problem(b, p);
    if (img == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "image must not be NULL");
    }
    batch_copy(b, img, static_cast<unsigned char*>(b.arena.p) + q.off_img, (size_t)q.v.nvox * sizeof(float));
    read_checks(*b.ctx);
  });
}

fir_status fir_batch_set_launch(fir_batch* batch, int block, int blocks_per_sm, int grab)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    if (block < 32 || block > 256 || block % 32 != 0)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "block size must be a multiple of 32 in [32, 256]");
    }
    if (blocks_per_sm < 0 || grab < 1 || grab > 64)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "blocks per SM must be >= 0 and grab in [1, 64]");
    }
    const int fit = batch_max_resident(block);
    const BatchLaunch s{block, blocks_per_sm > fit ? fit : blocks_per_sm, grab, b.shape.axial_tile};
    set_shape(b, s);
  });
}

fir_status fir_batch_set_bundle(fir_batch* batch, int axial_tile)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    if (axial_tile != 0 && axial_tile != 1 && axial_tile != 2 && axial_tile != 4 && axial_tile != 8)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "axial tile must be 0, 1, 2, 4 or 8");
    }
    BatchLaunch s = b.shape;
    s.axial_tile = axial_tile;
    set_shape(b, s);
  });
}

fir_status fir_batch_get_bundle(const fir_batch* batch, int* axial_tile)
{
  return guarded(__func__, [&] {
    if (batch == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "batch is NULL");
    }
    if (axial_tile != nullptr)
      *axial_tile = batch->shape.axial_tile;
  });
}

fir_status fir_batch_get_launch(const fir_batch* batch, int* block, int* blocks_per_sm, int* grab)
{
  return guarded(__func__, [&] {
    if (batch == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "batch is NULL");
    }
    if (block != nullptr)
      *block = batch->shape.block;
    if (blocks_per_sm != nullptr)
      *blocks_per_sm = batch->shape.blocks_per_sm;
    if (grab != nullptr)
      *grab = batch->shape.grab;
  });
}

fir_status fir_batch_schedule(const fir_batch* batch, int* n_steps, long long* n_launches)
{
  return guarded(__func__, [&] {
    if (batch == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "batch is NULL");
    }
    if (n_steps != nullptr)
      *n_steps = (int)batch->steps.size();
    if (n_launches != nullptr)
      *n_launches = batch->schedule_launches;
  });
}

fir_status fir_batch_tune(fir_batch* batch, double* best_ms)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    if (b.steps.empty())
    {
      if (best_ms != nullptr)
        *best_ms = 0.0;
      return;
    }
    // the first step whose projector batches problems (direct launches do
    // not use the shape)
    size_t t0 = 0;
    while (t0 < b.steps.size() && b.steps[t0].proj.n_items == 0)
    {
      ++t0;
    }
    if (t0 == b.steps.size())
    {
      b.tuned.clear();
      if (best_ms != nullptr)
        *best_ms = 0.0;
      return;
    }
    const BatchProblem* P = static_cast<const BatchProblem*>(b.desc.p);
    const BatchItem* I = static_cast<const BatchItem*>(b.items.p);
    int* queue = static_cast<int*>(b.queue.p);
    // linear bundles: every residency and grab; tiled bundles (A axial
    // planes x 32 / A tangential bins): one warp per bundle or a persistent
    // grid at full residency
    std::vector<BatchLaunch> cand;
    for (int tile : {0, 1, 2, 4})
    {
      for (int block : {64, 128, 256})
      {
        cand.push_back(BatchLaunch{block, 0, 1, tile});
        const int fit = batch_max_resident(block);
        for (int per_sm : {fit, std::max(1, fit / 2)})
        {
          for (int grab : {1, 2, 4})
          {
            if (tile == 0 || (per_sm == fit && grab == 1))
            {
              cand.push_back(BatchLaunch{block, per_sm, grab, tile});
            }
          }
        }
      }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cuda_ok(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_ok(cudaEventCreate(&e1), "cudaEventCreate");
    double best = 1e300;
    BatchLaunch pick = b.shape;
    const BatchLaunch start = b.shape;
    b.tuned.clear();
    try
    {
      batch_begin(b);
      for (const BatchLaunch& L : cand)
      {
        if (L.axial_tile != b.shape.axial_tile)
        {
          // the bundle form sets the projector's work units
          BatchLaunch s = b.shape;
          s.axial_tile = L.axial_tile;
          set_shape(b, s);
          P = static_cast<const BatchProblem*>(b.desc.p);
          I = static_cast<const BatchItem*>(b.items.p);
          queue = static_cast<int*>(b.queue.p);
        }
        double t_min = 1e300;
        for (int rep = 0; rep < 2; ++rep)
        {
          launch_batch_prepare(P, I + b.all.item_off, b.all.n_items, b.all.n_units, false, b.stream);
          check_launch(b.stream);
          cuda_ok(cudaMemsetAsync(queue, 0, sizeof(int), b.stream), "cudaMemsetAsync");
          cuda_ok(cudaEventRecord(e0, b.stream), "cudaEventRecord");
          batch_project(b, b.steps[t0].proj, queue, L, b.stream);
          cuda_ok(cudaEventRecord(e1, b.stream), "cudaEventRecord");
          cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize");
          float ms = 0.0f;
          cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
          t_min = std::min(t_min, (double)ms);
        }
        b.tuned.emplace_back(L, t_min);
        if (t_min < best)
        {
          best = t_min;
          pick = L;
        }
      }
      batch_end(b);
    }
    catch (...)
    {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      set_shape(b, start);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b.ctx->launches += (long long)cand.size() * 4;
    set_shape(b, pick);
    if (best_ms != nullptr)
    {
      *best_ms = best;
    }
    read_checks(*b.ctx);
  });
}

fir_status fir_batch_tune_report(const fir_batch* batch, int max, int* block, int* blocks_per_sm, int* grab,
                                 int* axial_tile, double* ms, int* n)
{
  return guarded(__func__, [&] {
    if (batch == nullptr)
    {
      fail(FIR_ERR_INVALID_ARGUMENT, "batch is NULL");
    }
    const int count = (int)batch->tuned.size();
    if (n != nullptr)
    {
      *n = count;
    }
    for (int i = 0; i < count && i < max; ++i)
    {
      const auto& t = batch->tuned[(size_t)i];
      if (block != nullptr)
        block[i] = t.first.block;
      if (blocks_per_sm != nullptr)
        blocks_per_sm[i] = t.first.blocks_per_sm;
      if (grab != nullptr)
        grab[i] = t.first.grab;
      if (axial_tile != nullptr)
        axial_tile[i] = t.first.axial_tile;
      if (ms != nullptr)
        ms[i] = t.second;
    }
  });
}

fir_status fir_batch_osem(fir_batch* batch, int use_graph)
{
  return guarded(__func__, [&] {
    fir_batch& b = check_batch(batch);
    batch_begin(b);
    if (use_graph)
    {
      if (b.exec == nullptr)
      {
        cuda_ok(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try
        {
          batch_enqueue(b, b.stream);
        }
        catch (...)
        {
          cudaGraph_t g = nullptr;
          cudaStreamEndCapture(b.stream, &g);
          if (g != nullptr)
          {
            cudaGraphDestroy(g);
          }
          cudaGetLastError();
          throw;
        }
        cuda_ok(cudaStreamEndCapture(b.stream, &b.graph), "cudaStreamEndCapture");
        cuda_ok(cudaGraphInstantiate(&b.exec, b.graph, 0), "cudaGraphInstantiate");
      }
      cuda_ok(cudaGraphLaunch(b.exec, b.stream), "cudaGraphLaunch");
    }
    else
    {
      batch_enqueue(b, b.stream);
    }
    batch_end(b);
    b.ctx->launches += b.schedule_launches;
  });
}

}  // extern "C"
