"""Deterministic backprojection (FIR_BACKPROJ_DETERMINISTIC).

Contributions are sorted per voxel into FIR's serial LOR order and summed with FIR's
rounding. The results must therefore be bit-identical to a single-threaded FIR run, and to
the oracle, which runs FIR's loops serially:
- backprojection;
- sensitivity;
- OSEM.

They must also not depend on the chunk size or on the run.
"""
import numpy as np
import pytest

from fir_b200 import capi, workloads
from fir_b200.geometry import OSEMParams

pytestmark = pytest.mark.gpu


def det_ctx(factory, scanner, chunk=0):
    ctx = factory(scanner)
    ctx.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
    if chunk:
        ctx.set_option(capi.FIR_OPT_DETERMINISTIC_CHUNK, chunk)
    return ctx


def test_backward_bit_identical_to_single_threaded_fir(gpu_ctx_factory, reference):
    w = workloads.small()
    reference.threads(1)
    y = np.random.default_rng(21).random(w.n_lors, dtype=np.float32)
    y[::5] = 0.0
    ctx = det_ctx(gpu_ctx_factory, w.scanner)
    for nsub in (1, 4):
        got = np.zeros(nsub * w.vol.n_voxels, np.float32)
        ctx.backward(w.proj, y, w.vol, got, nsub)
        want = reference.backward(w.scanner, w.proj, w.vol.with_frames(nsub), y, nsub)
        np.testing.assert_array_equal(got.reshape(want.shape), want)


def test_sensitivity_bit_identical_for_any_chunk(gpu_ctx_factory, restated):
    w = workloads.small()
    want = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    for chunk in (0, 5000, 123457):
        ctx = det_ctx(gpu_ctx_factory, w.scanner, chunk)
        got = np.zeros(4 * w.vol.n_voxels, np.float32)
        ctx.sensitivity(w.proj, w.vol, got, 4)
        np.testing.assert_array_equal(got.reshape(want.shape), want)


def test_osem_bit_identical_to_fir_and_reproducible(gpu_ctx_factory, restated):
    w = workloads.small()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 5)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    bias = np.full(w.n_lors, 0.03, np.float32)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=115.0)
    want = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    results = []
    for chunk in (0, 20000):
        ctx = det_ctx(gpu_ctx_factory, w.scanner, chunk)
        img = np.ones_like(x)
        ctx.osem(w.proj, y, w.vol, img, sens, prm, bias=bias)
        results.append(img)
    np.testing.assert_array_equal(results[0], want)
    np.testing.assert_array_equal(results[1], want)


def test_deterministic_ratio_backprojection_matches_atomic(gpu_ctx_factory):
    w = workloads.tiny()
    rng = np.random.default_rng(2)
    y = rng.random(w.n_lors, dtype=np.float32)
    img = (rng.random(w.vol.shape_zyx) + 0.5).astype(np.float32)
    a = np.zeros_like(img)
    b = np.zeros_like(img)
    gpu_ctx_factory(w.scanner).ratio_backprojection(w.proj, y, w.vol, img, a, 4, 1)
    det_ctx(gpu_ctx_factory, w.scanner).ratio_backprojection(w.proj, y, w.vol, img, b, 4, 1)
    assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b)
