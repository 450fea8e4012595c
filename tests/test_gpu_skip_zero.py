"""FIR_OPT_SKIP_ZERO_BINS: bins whose measured value is 0 are not traced.

Their ratio is exactly 0 in FIR's sub-iteration (reconAlgos.cc:152-157), so
their backprojection adds only zeros, and skipping them changes nothing but
the order of the float atomic additions.  The fused kernels take a compacted
list of the subset's non-zero bins.  Bars: one sub-iteration with and
without the option within 1e-6 relative L2, per voxel within 1e-5 of the
maximum; three OSEM iterations against the oracle within 1e-4.  Covered: the
exact traversal (exchanged double images), the opt-in float traversal, a
sinogram that is mostly zeros, and one that is all zeros; and the plain
backprojector (fir_backward), which takes the same list."""
import numpy as np
import pytest
import torch

from fir_b200 import capi, workloads

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def subiteration(ctx, w, y, sens, img0, subset, skip):
    ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, 1 if skip else 0)
    img = img0.clone()
    ctx.osem_subiteration(w.proj, y, w.vol, img, sens[subset], w.osem, subset, subset + 1)
    torch.cuda.synchronize()
    return img.cpu().numpy()


def sparse(y, keep, seed):
    """y with all but a fraction `keep` of its bins set to 0."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.where(torch.rand(y.shape, generator=g, device="cuda") < keep, y, torch.zeros_like(y))


@pytest.mark.parametrize("traversal", ["exact", "float"])
@pytest.mark.parametrize("keep", [1.0, 0.3, 0.0])
def test_skip_matches_full_enumeration(traversal, keep):
    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        if traversal == "float":
            ctx.set_option(capi.FIR_OPT_TRAVERSAL, capi.FIR_TRAVERSAL_FLOAT)
        y, sens = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
        y = sparse(y, keep, 3) if keep < 1.0 else y
        zeros = float((y == 0).double().mean())
        assert (keep == 1.0 and 0.0 < zeros < 0.9) or (keep < 1.0 and zeros >= 0.69)
        img0 = torch.rand(w.vol.shape_zyx, generator=torch.Generator(device="cuda").manual_seed(4),
                          device="cuda") + 0.5
        for subset in (0, w.osem.n_subsets - 1):
            want = subiteration(ctx, w, y, sens, img0, subset, False)
            got = subiteration(ctx, w, y, sens, img0, subset, True)
            if keep == 0.0:
                # nothing is backprojected: every voxel falls to 0 in the EM update
                assert not want.any() and not got.any()
                continue
            assert rel_l2(got, want) <= 1e-6, (subset, rel_l2(got, want))
            assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_skip_osem_matches_oracle(restated):
    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        y, sens = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
        ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, 1)
        assert ctx.get_option(capi.FIR_OPT_SKIP_ZERO_BINS) == 1
        img = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, img, sens, w.osem)
        torch.cuda.synchronize()
        got = img.cpu().numpy()
    want = restated.osem(w.scanner, w.proj, w.vol, y.cpu().numpy(), np.ones(w.vol.shape_zyx, np.float32),
                         sens.cpu().numpy(), w.osem)
    assert rel_l2(got, want) <= 1e-4


@pytest.mark.parametrize("keep", [1.0, 0.3])
def test_skip_backward_matches_full_enumeration(keep):
    """fir_backward of a measured sinogram, per subset, with and without the
    option (the plain backprojector takes the same compacted list)."""
    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        y, _ = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
        y = sparse(y, keep, 5) if keep < 1.0 else y
        nsub = w.osem.n_subsets
        out = []
        for skip in (0, 1):
            ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, skip)
            bp = torch.empty((nsub,) + tuple(w.vol.shape_zyx), device="cuda")
            ctx.backward(w.proj, y, w.vol, bp, nsub)
            torch.cuda.synchronize()
            out.append(bp.cpu().numpy())
    want, got = out
    assert float(want.max()) > 0
    assert rel_l2(got, want) <= 1e-6
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_skip_in_batch_matches_plain_osem():
    """A batch created on a context with the option skips zero bins in its
    batched projector (in place: a skipped lane idles); each problem matches
    fir_osem without the option within the float atomic order's 1e-5."""
    ws = [workloads.small(), workloads.tiny()]
    ctx = capi.Context(device=0)
    batch = None
    try:
        data, want = [], []
        for w in ws:
            ctx.set_scanner(w.scanner)
            y, sens = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
            y = sparse(y, 0.5, 9)
            img = torch.ones(w.vol.shape_zyx, device="cuda")
            ctx.osem(w.proj, y, w.vol, img, sens, w.osem)
            torch.cuda.synchronize()
            data.append((y, sens))
            want.append(img.cpu().numpy())
        ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, 1)
        batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem) for w in ws])
        for k, w in enumerate(ws):
            batch.set_data(k, *data[k])
            batch.set_image(k, np.ones(w.vol.shape_zyx, np.float32))
        batch.osem(use_graph=True)
        for k in range(len(ws)):
            assert rel_l2(batch.get_image(k), want[k]) <= 1e-5, k
    finally:
        if batch is not None:
            batch.close()
        ctx.close()
