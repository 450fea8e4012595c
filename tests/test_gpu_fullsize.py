"""The clinical workload at full size (32 rings x 512 crystals, 200x200x64
image at 3 mm; 3.28e7 LORs, and 1.34e8 in its full-FOV form) against FIR
itself, compiled from its sources and run on the host's cores:
* the forward projection of the phantom equals FIR's on every bin, in both
  forms;
* one full OSEM iteration (16 subsets, FWHM 4 mm filter, cut radius) from
  the same data and sensitivity agrees with FIR's to 1e-4 relative L2.
"""
import os

import numpy as np
import pytest
import torch

from fir_b200 import workloads

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def clinical(gpu_ctx_factory, reference):
    reference.threads(os.cpu_count() or 1)
    w = workloads.clinical()
    ctx = gpu_ctx_factory(w.scanner)
    return w, ctx


def test_clinical_forward_bit_identical_to_fir(clinical, reference):
    w, ctx = clinical
    x = workloads.activity(w)
    got = torch.empty(w.n_lors, device=DEV)
    ctx.forward(w.vol, torch.from_numpy(x).to(DEV), w.proj, got)
    torch.cuda.synchronize()
    want = reference.forward(w.scanner, w.proj, w.vol, x, w.n_lors)
    np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_clinical_osem_iteration_matches_fir(clinical, reference):
    from fir_b200.geometry import OSEMParams

    w, ctx = clinical
    y, sens = workloads.measured_on_gpu(ctx, w, DEV, attenuation=True)
    prm = OSEMParams(n_iterations=1, n_subsets=16, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=290.0)
    img = torch.ones(w.vol.shape_zyx, device=DEV)
    ctx.osem(w.proj, y, w.vol, img, sens, prm)
    torch.cuda.synchronize()
    got = img.cpu().numpy()
    want = reference.osem(w.scanner, w.proj, w.vol, y.cpu().numpy(), np.ones(w.vol.shape_zyx, np.float32),
                          sens.cpu().numpy(), prm)
    assert float(want.max()) > 0
    assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want)


def test_clinical_full_fov_forward_bit_identical_to_fir(gpu_ctx_factory, reference):
    """All 511 tangential bins (1.34e8 LORs, the '~1e8 LORs' form of the
    clinical configuration): every bin equals FIR's."""
    reference.threads(os.cpu_count() or 1)
    w = workloads.clinical(full_fov=True)
    ctx = gpu_ctx_factory(w.scanner)
    x = workloads.activity(w)
    got = torch.empty(w.n_lors, device=DEV)
    ctx.forward(w.vol, torch.from_numpy(x).to(DEV), w.proj, got)
    torch.cuda.synchronize()
    want = reference.forward(w.scanner, w.proj, w.vol, x, w.n_lors)
    np.testing.assert_array_equal(got.cpu().numpy(), want)
