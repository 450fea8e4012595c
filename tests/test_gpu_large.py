"""The large workload (64 rings x 640 crystals, 2.1e8 LORs, 320x320x128 at
1.5 mm, exact geometry) at full size.

FIR itself is invalid here: it truncates 1.5 mm extents to 1 mm, and its
16-bit crystal ids overflow.  The oracle is therefore the C restatement with
real extents:
* on a random sample of 4000 LORs, index lists and lengths are bit-identical,
  and so is each sampled bin of the full forward projection (FIR's float
  accumulation replayed along the oracle's paths);
* on all LORs, the adjoint test holds, and so does exact linearity under
  scaling by two;
* one OSEM iteration (32 subsets) run as one captured graph (a batch of one
  problem) matches fir_osem within 1e-5 relative L2;
* the volume's double copy does not fit in L2 beside the accumulator, so the
  fused kernel gathers the float image, in two launches that each take the
  LORs of one orientation with their own (x/y-exchanged) image and
  accumulator: one subset's backprojected ratio matches the deterministic
  mode, which gathers the double copy and sums in FIR's order, within the
  1e-6 relative L2 of float atomic order.
"""
import numpy as np
import pytest
import torch

from fir_b200 import capi, workloads
from test_gpu_parity import assert_paths_equal, lor_ends

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def large():
    w = workloads.large()
    ctx = capi.Context(w.scanner)
    ctx.set_option(capi.FIR_OPT_GEOMETRY, capi.FIR_GEOMETRY_EXACT)
    yield w, ctx
    ctx.close()


def test_sampled_paths_and_projections_bit_exact(large, restated):
    w, ctx = large
    rng = np.random.default_rng(8)
    bins = np.sort(rng.choice(w.n_lors, 4000, replace=False))
    got = ctx.lor_paths(w.proj, w.vol, bins)
    want = restated.siddon_paths(w.vol, lor_ends(restated, w, bins), truncate=False)
    assert_paths_equal(got, want)
    # forward projection of the phantom at the sampled bins
    x = workloads.activity(w)
    y = torch.empty(w.n_lors, device=DEV)
    ctx.forward(w.vol, torch.from_numpy(x).to(DEV), w.proj, y)
    _, counts, coords, lengths = want
    xf = x.ravel().astype(np.float64)
    line = np.zeros(bins.size, np.float32)
    for k in range(coords.shape[1]):
        on = counts > k
        if not on.any():
            break
        c = np.where(on, coords[:, k], 0)
        upd = (line.astype(np.float64) + lengths[:, k] * xf[c]).astype(np.float32)
        line = np.where(on, upd, line)
    np.testing.assert_array_equal(y.cpu().numpy()[bins], line)


def test_full_size_adjoint_and_linearity(large):
    w, ctx = large
    g = torch.Generator(device=DEV).manual_seed(3)
    x = torch.rand(w.vol.shape_zyx, generator=g, device=DEV)
    y = torch.rand(w.n_lors, generator=g, device=DEV)
    ax = torch.empty(w.n_lors, device=DEV)
    ctx.forward(w.vol, x, w.proj, ax)
    aty = torch.empty(w.vol.shape_zyx, device=DEV)
    ctx.backward(w.proj, y, w.vol, aty, 1)
    lhs = float(torch.dot(ax.double(), y.double()))
    rhs = float(torch.dot(x.double().ravel(), aty.double().ravel()))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    ax2 = torch.empty_like(ax)
    ctx.forward(w.vol, x * 2, w.proj, ax2)
    assert torch.equal(ax2, ax * 2)


def test_one_iteration_graph_matches_plain(large):
    w, ctx = large
    y, sens = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
    plain = torch.ones(w.vol.shape_zyx, device=DEV)
    ctx.osem(w.proj, y, w.vol, plain, sens, w.osem)
    batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem)])
    batch.set_data(0, y, sens)
    batch.set_image(0, np.ones(w.vol.shape_zyx, np.float32))
    assert batch.schedule()[0] == w.osem.n_iterations * w.osem.n_subsets
    batch.osem(use_graph=True)
    got = batch.get_image(0)
    want = plain.cpu().numpy()
    assert np.isfinite(got).all() and float(want.max()) > 0
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
    batch.close()


def test_float_gather_subset_matches_deterministic(large):
    w, ctx = large
    g = torch.Generator(device=DEV).manual_seed(5)
    img = torch.rand(w.vol.shape_zyx, generator=g, device=DEV) + 0.5
    y = torch.poisson(torch.full((w.n_lors,), 3.0, device=DEV), generator=g)
    got = torch.zeros_like(img)
    ctx.ratio_backprojection(w.proj, y, w.vol, img, got, w.osem.n_subsets, 3)
    det = capi.Context(w.scanner)
    det.set_option(capi.FIR_OPT_GEOMETRY, capi.FIR_GEOMETRY_EXACT)
    det.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
    want = torch.zeros_like(img)
    det.ratio_backprojection(w.proj, y, w.vol, img, want, w.osem.n_subsets, 3)
    torch.cuda.synchronize()
    det.close()
    assert float(want.max()) > 0
    rel = float((got.double() - want.double()).norm() / want.double().norm())
    assert rel <= 1e-6
