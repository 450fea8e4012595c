"""The opt-in float traversal (FIR_OPT_TRAVERSAL = FIR_TRAVERSAL_FLOAT).

It is not FIR's arithmetic: the oracle's precision study shows its voxel lists
differing from FIR's for a few per cent of LORs.  What it must keep is the
reconstruction: OSEM images within 1e-4 relative L2 of the exact traversal's
(small workload, 3 iterations of 4 subsets against the oracle; clinical
workload, one iteration of 16 subsets against the exact mode).  The option is
validated and reads back, and deterministic mode keeps the exact traversal."""
import numpy as np
import pytest
import torch

from fir_b200 import capi, workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _data(ctx, w):
    return workloads.measured_on_gpu(ctx, w, torch.device("cuda", 0), attenuation=True)


def test_float_traversal_osem_small_matches_oracle(restated):
    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        y, sens = _data(ctx, w)
        ctx.set_option(capi.FIR_OPT_TRAVERSAL, capi.FIR_TRAVERSAL_FLOAT)
        assert ctx.get_option(capi.FIR_OPT_TRAVERSAL) == capi.FIR_TRAVERSAL_FLOAT
        img = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, img, sens, w.osem)
        torch.cuda.synchronize()
        got = img.cpu().numpy()
    want = restated.osem(w.scanner, w.proj, w.vol, y.cpu().numpy(), np.ones(w.vol.shape_zyx, np.float32),
                         sens.cpu().numpy(), w.osem)
    err = rel_l2(got, want)
    assert 0.0 < err <= 1e-4, err


def test_float_traversal_osem_clinical_iteration():
    w = workloads.clinical()
    with capi.Context(w.scanner) as ctx:
        y, sens = _data(ctx, w)
        prm = w.osem
        one = type(prm)(n_iterations=1, n_subsets=prm.n_subsets, convolution_interval=prm.convolution_interval,
                        fwhm_xyz=list(prm.fwhm_xyz), cut_radius=prm.cut_radius)
        exact = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, exact, sens, one)
        ctx.set_option(capi.FIR_OPT_TRAVERSAL, capi.FIR_TRAVERSAL_FLOAT)
        fast = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, fast, sens, one)
        torch.cuda.synchronize()
        err = rel_l2(fast.cpu().numpy(), exact.cpu().numpy())
    assert 0.0 < err <= 1e-4, err


def test_float_traversal_option_checks():
    w = workloads.tiny()
    with capi.Context(w.scanner) as ctx:
        with pytest.raises(capi.FirError):
            ctx.set_option(capi.FIR_OPT_TRAVERSAL, 7)
        assert ctx.get_option(capi.FIR_OPT_TRAVERSAL) == capi.FIR_TRAVERSAL_EXACT
        # deterministic backprojection keeps FIR's traversal: bit-identical runs
        y, sens = _data(ctx, w)
        ctx.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
        a = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, a, sens, w.osem)
        ctx.set_option(capi.FIR_OPT_TRAVERSAL, capi.FIR_TRAVERSAL_FLOAT)
        b = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, b, sens, w.osem)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
