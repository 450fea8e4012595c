"""The x/y-exchanged images, on volumes that are not square.

LORs that run mostly along x are traced in a copy of the image with x and y
exchanged ([z][x][y]), and their backprojection accumulates in such a copy
that is then added back.  A square volume cannot tell nx from ny, so these
cases use unequal, odd sizes (wider in x, and wider in y) that are not
multiples of the 32-voxel tiles of the exchange kernels.  The bars are those
of the other parity tests:
  * forward projections (single- and multi-frame): bit-identical to the oracle;
  * backprojection and sensitivity: relative L2 <= 1e-6, per voxel <= 1e-5 of
    the maximum;
  * OSEM, plain and batched: relative L2 <= 1e-4 against the oracle.
A mid-size volume that only fits L2 as float image and accumulator, one
orientation at a time, runs the fused kernel as two launches; it is checked
against the deterministic mode (1e-6 relative L2) and, batched beside a small
problem, against fir_osem (1e-5).
"""
import numpy as np
import pytest
import torch

from fir_b200 import capi, workloads
from fir_b200.geometry import OSEMParams, ProjSpec, ScannerSpec, VolSpec

pytestmark = pytest.mark.gpu

VOLS = {
    "wide_x": VolSpec.centred((45, 38, 11), (4.0, 4.0, 4.0)),
    "wide_y": VolSpec.centred((27, 52, 9), (3.0, 3.0, 4.0)),
}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def assert_scatter_close(got, want):
    assert rel_l2(got, want) <= 1e-6
    assert float(np.max(np.abs(np.asarray(got, np.float64) - want))) <= 1e-5 * float(np.max(np.abs(want)))


def geometry():
    scanner = ScannerSpec.ring(6, 128, 150.0, 4.0)
    proj = ProjSpec(6, 128, 11, workloads.n_tang_for_fov(128, 150.0, 100.0))
    return scanner, proj


def image(v, seed):
    return (np.random.default_rng(seed).random(v.shape_zyx, dtype=np.float32) + 0.25).astype(np.float32)


@pytest.mark.parametrize("name", sorted(VOLS))
def test_forward_bit_exact(gpu_ctx_factory, restated, name):
    v = VOLS[name]
    s, p = geometry()
    x = image(v, 1)
    ctx = gpu_ctx_factory(s)
    got = np.zeros(capi.proj_geometry(p)["n_bins"], np.float32)
    ctx.forward(v, x, p, got)
    np.testing.assert_array_equal(got, restated.forward(s, p, v, x))


@pytest.mark.parametrize("name", sorted(VOLS))
def test_backward_and_sensitivity(gpu_ctx_factory, restated, name):
    v = VOLS[name]
    s, p = geometry()
    nb = capi.proj_geometry(p)["n_bins"]
    y = np.random.default_rng(2).random(nb, dtype=np.float32)
    ctx = gpu_ctx_factory(s)
    for nsub in (1, 4):
        bp = np.zeros(nsub * v.n_voxels, np.float32)
        ctx.backward(p, y, v, bp, nsub)
        assert_scatter_close(bp.reshape(-1, *v.shape_zyx[1:]), restated.backward(s, p, v, y, nsub))
    sens = np.zeros(4 * v.n_voxels, np.float32)
    ctx.sensitivity(p, v, sens, 4)
    assert_scatter_close(sens.reshape(-1, *v.shape_zyx[1:]), restated.sensitivity(s, p, v, 4))


def osem_case(restated, v, seed):
    s, p = geometry()
    x = image(v, seed)
    y = workloads.poisson_counts(restated.forward(s, p, v, x), 2e5, seed)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0])
    sens = restated.sensitivity(s, p, v, prm.n_subsets)
    want = restated.osem(s, p, v, y, np.ones_like(x), sens, prm)
    return s, p, prm, y, sens, want


@pytest.mark.parametrize("name", sorted(VOLS))
def test_osem_matches_oracle(gpu_ctx_factory, restated, name):
    v = VOLS[name]
    s, p, prm, y, sens, want = osem_case(restated, v, 3)
    ctx = gpu_ctx_factory(s)
    img = np.ones(v.shape_zyx, np.float32)
    ctx.osem(p, y, v, img, sens, prm)
    assert rel_l2(img, want) <= 1e-4


def test_batched_osem_matches_oracle(restated):
    cases = [(v,) + osem_case(restated, v, 4 + k) for k, v in enumerate(VOLS[n] for n in sorted(VOLS))]
    ctx = capi.Context(device=0)
    batch = capi.Batch(ctx, [(s, p, v, prm) for v, s, p, prm, *_ in cases])
    try:
        for k, (v, s, p, prm, y, sens, want) in enumerate(cases):
            batch.set_data(k, y, sens)
            batch.set_image(k, np.ones(v.shape_zyx, np.float32))
        batch.osem(use_graph=False)
        for k, (v, s, p, prm, y, sens, want) in enumerate(cases):
            assert rel_l2(batch.get_image(k), want) <= 1e-4, k
    finally:
        batch.close()
        ctx.close()


@pytest.mark.parametrize("name", sorted(VOLS))
def test_frames_match_single_frame(gpu_ctx_factory, name):
    v = VOLS[name]
    s, p = geometry()
    nb = capi.proj_geometry(p)["n_bins"]
    ctx = gpu_ctx_factory(s)
    g = torch.Generator(device="cuda").manual_seed(5)
    for n in (2, 4):
        x = torch.rand((n,) + tuple(v.shape_zyx), generator=g, device="cuda")
        y = torch.empty(n, nb, device="cuda")
        ctx.forward_frames(v.with_frames(n), x, p, y)
        q = torch.rand(n, nb, generator=g, device="cuda")
        b = torch.empty((n,) + tuple(v.shape_zyx), device="cuda")
        ctx.backward_frames(p, q, v.with_frames(n), b)
        for f in range(n):
            want = torch.empty(nb, device="cuda")
            ctx.forward(v, x[f].contiguous(), p, want)
            assert torch.equal(y[f], want), (n, f)
            wb = torch.empty(tuple(v.shape_zyx), device="cuda")
            ctx.backward(p, q[f].contiguous(), v, wb, 1)
            torch.cuda.synchronize()
            assert_scatter_close(b[f].cpu().numpy(), wb.cpu().numpy().astype(np.float64))


def mid_volume():
    """A volume whose double copy and accumulator (12 B per voxel) overflow the
    device's L2 while the float image and accumulator (8 B) fit: the fused
    kernel then gathers floats, in two launches, one per orientation, each
    with its own (exchanged) float image and accumulator.  Unequal sizes, not
    multiples of the 32-voxel tiles; sub-millimetre voxels, so exact geometry."""
    l2 = torch.cuda.get_device_properties(0).L2_cache_size
    nx, ny = 331, 287
    nz = int(round(l2 / 9.5 / (nx * ny)))
    n = nx * ny * nz
    assert 8 * n <= l2 < 12 * n
    return VolSpec.centred((nx, ny, nz), (0.3, 0.3, 24.0 / nz))


def test_mid_volume_orientation_launches_match_deterministic():
    """One subset's backprojected ratio from the two orientation launches
    against the deterministic mode (double copy, one orientation, FIR's
    summation order): within the float atomic order's 1e-6 relative L2."""
    v = mid_volume()
    s, p = geometry()
    nb = capi.proj_geometry(p)["n_bins"]
    g = torch.Generator(device="cuda").manual_seed(7)
    img = torch.rand(v.shape_zyx, generator=g, device="cuda") + 0.5
    y = torch.poisson(torch.full((nb,), 3.0, device="cuda"), generator=g)
    got = torch.zeros_like(img)
    want = torch.zeros_like(img)
    ctx = capi.Context(s)
    det = capi.Context(s)
    try:
        for c in (ctx, det):
            c.set_option(capi.FIR_OPT_GEOMETRY, capi.FIR_GEOMETRY_EXACT)
        det.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
        ctx.ratio_backprojection(p, y, v, img, got, 4, 1)
        det.ratio_backprojection(p, y, v, img, want, 4, 1)
        torch.cuda.synchronize()
    finally:
        det.close()
        ctx.close()
    assert float(want.max()) > 0
    assert_scatter_close(got.cpu().numpy(), want.cpu().numpy().astype(np.float64))


def test_mid_volume_batched_osem_matches_plain():
    """In a batch, the mid-size problem runs fir_osem's kernel in launches of
    its own (two per step, one per orientation) beside the batched projector
    of a small problem: one OSEM iteration of both, tuned and captured as a
    graph, against fir_osem on each."""
    vols = [mid_volume(), VOLS["wide_x"]]
    s, p = geometry()
    nb = capi.proj_geometry(p)["n_bins"]
    prm = OSEMParams(n_iterations=1, n_subsets=4, convolution_interval=1, fwhm_xyz=[1.0, 1.0, 1.0])
    ctx = capi.Context(s)
    ctx.set_option(capi.FIR_OPT_GEOMETRY, capi.FIR_GEOMETRY_EXACT)
    batch = None
    try:
        data, want = [], []
        for k, v in enumerate(vols):
            x = torch.rand(v.shape_zyx, generator=torch.Generator(device="cuda").manual_seed(8 + k), device="cuda")
            ax = torch.empty(nb, device="cuda")
            ctx.forward(v, x, p, ax)
            y = torch.poisson(ax * (2e6 / float(ax.double().sum())))
            sens = torch.empty((prm.n_subsets,) + tuple(v.shape_zyx), device="cuda")
            ctx.sensitivity(p, v, sens, prm.n_subsets)
            plain = torch.ones(v.shape_zyx, device="cuda")
            ctx.osem(p, y, v, plain, sens, prm)
            data.append((y, sens))
            want.append(plain.cpu().numpy())
        batch = capi.Batch(ctx, [(s, p, v, prm) for v in vols])
        for k, v in enumerate(vols):
            batch.set_data(k, *data[k])
            batch.set_image(k, np.ones(v.shape_zyx, np.float32))
        n_steps, launches = batch.schedule()
        # prepare, then per sub-iteration: the batched projector, two direct
        # projector launches, the EM update and the three filter passes
        assert (n_steps, launches) == (prm.n_subsets, 1 + prm.n_subsets * 7)
        assert batch.tune() > 0 and len(batch.tune_report()) == 39
        batch.osem(use_graph=True)
        for k, v in enumerate(vols):
            got = batch.get_image(k)
            assert np.isfinite(got).all() and float(want[k].max()) > 0
            assert rel_l2(got, want[k]) <= 1e-5, k
    finally:
        if batch is not None:
            batch.close()
        ctx.close()
