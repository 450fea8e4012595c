"""Batched OSEM (fir_batch_*): many problems of uneven sizes in one schedule.

Each problem of a batch must reconstruct as fir_osem does on it alone.  The
two differ only in the order of the float atomic additions of the
backprojection, so the images agree to 1e-5 relative L2.  Against the oracle
the bar is the 1e-4 relative L2 of OSEM parity.

The CUDA graph replay, the direct launches and every launch shape (plain or
persistent, any grab, linear or tiled LOR bundles) must give the same images
within the same tolerance.
"""
import numpy as np
import pytest
import torch

from fir_b200 import capi, workloads
from fir_b200.geometry import OSEMParams, ProjSpec, ScannerSpec, VolSpec

pytestmark = pytest.mark.gpu

TOL_ATOMIC = 1e-5
TOL_ORACLE = 1e-4


def mixed_problems():
    """Five problems: different scanners, images, subsets, iterations, with and
    without filter and cut; one carries a bias sinogram."""
    rows = [
        # rings, crystals, radius, nxy, nz, voxel, subsets, iterations, fwhm, cut
        (4, 96, 150.0, 32, 8, 4.0, 4, 2, 4.0, 0.0),
        (6, 128, 200.0, 48, 12, 3.0, 2, 2, 0.0, 60.0),
        (5, 112, 180.0, 40, 10, 2.0, 4, 1, 4.0, 35.0),
        (8, 160, 250.0, 64, 16, 4.0, 8, 1, 4.0, 110.0),
        (4, 104, 160.0, 36, 9, 3.0, 2, 3, 0.0, 0.0),
    ]
    out = []
    for i, (nr, nc, rad, nxy, nz, vox, nsub, nit, fwhm, cut) in enumerate(rows):
        fov = min(0.9 * nxy * vox / 2, 0.7 * rad)
        prm = OSEMParams(n_iterations=nit, n_subsets=nsub, convolution_interval=1 if fwhm > 0 else 0,
                         fwhm_xyz=[fwhm, fwhm, fwhm], cut_radius=cut)
        out.append(workloads.Workload(
            name=f"mixed{i}", scanner=ScannerSpec.ring(nr, nc, rad, 4.0),
            proj=ProjSpec(nr, nc, 2 * nr - 1, workloads.n_tang_for_fov(nc, rad, fov)),
            vol=VolSpec.centred((nxy, nxy, nz), (vox, vox, vox)), osem=prm, counts=2e5, seed=100 + i,
            kind="cylinder", extra={"cyl_radius": 0.7 * fov}))
    return out


def build(ws, bias_for=(3,)):
    dev = torch.device("cuda", 0)
    ctx = capi.Context(device=0)
    data = []
    for k, w in enumerate(ws):
        ctx.set_scanner(w.scanner)
        y, sens = workloads.measured_on_gpu(ctx, w, dev, attenuation=False)
        bias = torch.full_like(y, 0.05) if k in bias_for else None
        data.append((y, sens, bias))
    torch.cuda.synchronize()
    batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem) for w in ws])
    for k, (y, sens, bias) in enumerate(data):
        batch.set_data(k, y, sens, bias)
    return ctx, batch, data


def reset(batch, ws):
    for k, w in enumerate(ws):
        batch.set_image(k, np.ones(w.vol.shape_zyx, np.float32))


def plain(ws, data):
    out = []
    for w, (y, sens, bias) in zip(ws, data):
        ctx = capi.Context(w.scanner, device=0)
        img = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, img, sens, w.osem, bias=bias)
        torch.cuda.synchronize()
        out.append(img.cpu().numpy())
        ctx.close()
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_batch_matches_plain_osem_per_problem():
    ws = mixed_problems()
    ctx, batch, data = build(ws)
    want = plain(ws, data)
    n_steps, launches = batch.schedule()
    assert n_steps == max(w.osem.n_iterations * w.osem.n_subsets for w in ws)
    for use_graph in (False, True):
        reset(batch, ws)
        batch.osem(use_graph=use_graph)
        for k, w in enumerate(ws):
            got = batch.get_image(k)
            assert rel(got, want[k]) <= TOL_ATOMIC, (use_graph, k, rel(got, want[k]))
    # graph replay: a second run from the same start gives the same images
    reset(batch, ws)
    batch.osem(use_graph=True)
    for k in range(len(ws)):
        assert rel(batch.get_image(k), want[k]) <= TOL_ATOMIC
    batch.close()
    ctx.close()


@pytest.mark.parametrize("shape", [(128, 0, 1), (64, 4, 1), (256, 2, 4), (128, 64, 2)])
def test_launch_shapes_agree(shape):
    ws = mixed_problems()[:3]
    ctx, batch, data = build(ws, bias_for=())
    want = plain(ws, data)
    batch.set_launch(*shape)
    blk, per_sm, grab = batch.launch()
    assert blk == shape[0] and grab == shape[2] and 0 <= per_sm <= shape[1]
    reset(batch, ws)
    batch.osem(use_graph=True)
    for k in range(len(ws)):
        assert rel(batch.get_image(k), want[k]) <= TOL_ATOMIC
    batch.close()
    ctx.close()


@pytest.mark.parametrize("tile,shape", [(1, (128, 0, 1)), (2, (64, 0, 1)), (4, (128, 64, 1)), (8, (256, 2, 2))])
def test_bundle_shapes_agree(tile, shape):
    """Tiled bundles (tile axial planes x 32 / tile tangential bins, padded
    at the planes' edges) cover every LOR once: same images as fir_osem."""
    ws = mixed_problems()
    ctx, batch, data = build(ws)
    want = plain(ws, data)
    batch.set_launch(*shape)
    batch.set_bundle(tile)
    assert batch.bundle() == tile
    reset(batch, ws)
    batch.osem(use_graph=True)
    for k in range(len(ws)):
        assert rel(batch.get_image(k), want[k]) <= TOL_ATOMIC, (tile, k)
    # back to linear bundles: the schedule is rebuilt
    batch.set_bundle(0)
    reset(batch, ws)
    batch.osem(use_graph=False)
    for k in range(len(ws)):
        assert rel(batch.get_image(k), want[k]) <= TOL_ATOMIC
    batch.close()
    ctx.close()


def test_bundle_shape_checked():
    ws = mixed_problems()[:1]
    ctx, batch, data = build(ws, bias_for=())
    for bad in (3, 16, -1):
        with pytest.raises(capi.FirError, match="axial tile"):
            batch.set_bundle(bad)
    assert batch.bundle() == 0
    batch.close()
    ctx.close()


def test_tuner_keeps_images_and_results(restated):
    ws = mixed_problems()[:2]
    ctx, batch, data = build(ws, bias_for=())
    reset(batch, ws)
    ms = batch.tune()
    assert ms > 0
    blk, per_sm, grab = batch.launch()
    assert blk in (64, 128, 256) and grab in (1, 2, 4)
    assert batch.bundle() in (0, 1, 2, 4)
    table = batch.tune_report()
    assert len(table) == 3 * 7 + 3 * 3 * 2 and min(t[-1] for t in table) == pytest.approx(ms)
    assert {t[3] for t in table} == {0, 1, 2, 4}
    # the tuner leaves the starting images alone
    for k, w in enumerate(ws):
        np.testing.assert_array_equal(batch.get_image(k), np.ones(w.vol.shape_zyx, np.float32))
    batch.osem(use_graph=True)
    for k, (w, (y, sens, _)) in enumerate(zip(ws, data)):
        want = restated.osem(w.scanner, w.proj, w.vol, y.cpu().numpy(), np.ones(w.vol.shape_zyx, np.float32),
                             sens.cpu().numpy(), w.osem)
        assert rel(batch.get_image(k), want) <= TOL_ORACLE
    batch.close()
    ctx.close()


def test_batch_errors():
    ws = mixed_problems()[:2]
    ctx = capi.Context(device=0)
    batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem) for w in ws])
    with pytest.raises(capi.FirError, match="out of range"):
        batch.set_image(2, np.ones(4, np.float32))
    with pytest.raises(capi.FirError, match="multiple of 32"):
        batch.set_launch(100, 1, 1)
    with pytest.raises(capi.FirError, match="grab"):
        batch.set_launch(128, 1, 0)
    bad = OSEMParams(n_iterations=1, n_subsets=5)
    with pytest.raises(capi.FirError, match="divisor"):
        capi.Batch(ctx, [(ws[0].scanner, ws[0].proj, ws[0].vol, bad)])
    with pytest.raises(capi.FirError, match="same number of rings"):
        capi.Batch(ctx, [(ws[1].scanner, ws[0].proj, ws[0].vol, ws[0].osem)])
    batch.close()
    ctx.close()


def test_problem_with_large_subsets_runs_single_problem_kernel():
    """A problem with 2^22 or more LORs per subset (the clinical scanner, 4
    subsets) is not batched: each step runs fir_osem's kernel for it, with its
    descriptor as kernel parameters, beside the batched launch of a small
    problem.  Both images match fir_osem, as a graph and as direct launches,
    and a new bias sinogram reaches the single-problem launches of the next
    graph (the captured graph holds the old pointer, so it is rebuilt)."""
    base = workloads.clinical()
    big = workloads.Workload(
        name="wide_subsets", scanner=base.scanner, proj=base.proj,
        vol=VolSpec.centred((64, 64, 16), (4.0, 4.0, 4.0)),
        osem=OSEMParams(n_iterations=1, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
        counts=2e6, seed=7, kind="cylinder", extra={"cyl_radius": 80.0})
    assert capi.proj_geometry(big.proj)["n_bins"] // big.osem.n_subsets >= 1 << 22
    ws = [big, mixed_problems()[0]]
    ctx, batch, data = build(ws, bias_for=(0,))
    try:
        n_steps, launches = batch.schedule()
        # prepare; per step: the batched projector (small problem, steps 1..8),
        # the single-problem projector (big problem, steps 1..4), EM, filter
        small = ws[1].osem.n_iterations * ws[1].osem.n_subsets
        assert n_steps == small
        assert launches == 1 + big.osem.n_subsets * (1 + 1 + 1 + 3) + (small - big.osem.n_subsets) * (1 + 1 + 3)
        want = plain(ws, data)
        for use_graph in (True, False):
            reset(batch, ws)
            batch.osem(use_graph=use_graph)
            for k in range(len(ws)):
                got = batch.get_image(k)
                assert rel(got, want[k]) <= TOL_ATOMIC, (use_graph, k)
        y, sens, _ = data[0]
        bias = torch.full_like(y, 0.2)
        batch.set_data(0, y, sens, bias)
        want0 = plain([big], [(y, sens, bias)])[0]
        reset(batch, ws)
        batch.osem(use_graph=True)
        assert rel(batch.get_image(0), want0) <= TOL_ATOMIC
        assert rel(want0, want[0]) > 10 * TOL_ATOMIC  # the new bias changes the image
    finally:
        batch.close()
        ctx.close()
