"""Parity of the sm_100a path with the CPU oracle, through the C ABI.

Bars (fixed here, per operation):
  * Siddon index lists and lengths, forward projections, attenuation factors,
    Gaussian filter, cut, mask, HU->mu, sinogram exp/product, EM update:
    bit-identical to the oracle (which is bit-identical to FIR).
  * Backprojection and sensitivity (float atomics, order-dependent like FIR's
    "omp atomic"): relative L2 error <= 1e-6 and per-voxel error <= 1e-5 of the
    image maximum.
  * OSEM images after the stated iterations: relative L2 error <= 1e-4.
"""
import os

import numpy as np
import pytest

from fir_b200 import capi, workloads
from fir_b200.geometry import OSEMParams, ProjSpec, ScannerSpec, VolSpec

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch as t

    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    return t


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def assert_scatter_close(got, want):
    assert rel_l2(got, want) <= 1e-6
    assert float(np.max(np.abs(np.asarray(got, np.float64) - want))) <= 1e-5 * float(np.max(np.abs(want)))


def assert_paths_equal(got, want):
    """Equal crossing flags and element counts, and bit-identical index and
    length lists; slots past a path's last element are not part of the
    output and are not compared."""
    c1, n1, co1, le1 = got
    c2, n2, co2, le2 = want
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(n1, n2)
    cap = min(co1.shape[1], co2.shape[1])
    mask = np.arange(cap)[None, :] < np.minimum(n1, cap)[:, None]
    np.testing.assert_array_equal(co1[:, :cap][mask], co2[:, :cap][mask])
    np.testing.assert_array_equal(le1[:, :cap][mask], le2[:, :cap][mask])


def lor_ends(restated, w, bins):
    """Oracle end points of flat-order bins."""
    xy, z = restated.scanner_tables(w.scanner)
    table = restated.lor_table_bins(w.proj, bins)
    return np.stack([xy[2 * table[:, 1]], xy[2 * table[:, 1] + 1], z[table[:, 0]],
                     xy[2 * table[:, 3]], xy[2 * table[:, 3] + 1], z[table[:, 2]]], axis=1)


# ------------------------------------------------------------ Siddon paths

@pytest.mark.parametrize("name", ["unit3x3x2", "unit512x384"])
def test_golden_paths_bit_exact(gpu_ctx_factory, name):
    g = np.load(os.path.join(GOLDEN, "siddon_cases.npz"))
    a = g[name + "_vol"]
    v = VolSpec(tuple(int(x) for x in a[0:3]), tuple(a[3:6]), tuple(a[6:9]))
    ctx = gpu_ctx_factory()
    got = ctx.siddon_paths(v, g[name + "_segs"], cap=g[name + "_coords"].shape[1])
    assert_paths_equal(got, tuple(g[name + k] for k in ("_crosses", "_counts", "_coords", "_lengths")))


@pytest.mark.parametrize("wname", ["small", "clinical"])
def test_lor_paths_bit_exact(gpu_ctx_factory, restated, wname):
    w = getattr(workloads, wname)()
    nb = w.n_lors
    rng = np.random.default_rng(5)
    bins = np.arange(nb) if nb <= 200_000 else np.sort(rng.choice(nb, 20_000, replace=False))
    ctx = gpu_ctx_factory(w.scanner)
    got = ctx.lor_paths(w.proj, w.vol, bins)
    assert_paths_equal(got, restated.siddon_paths(w.vol, lor_ends(restated, w, bins)))


def test_random_segments_bit_exact_both_geometries(gpu_ctx_factory, restated):
    rng = np.random.default_rng(17)
    v = VolSpec((40, 44, 20), (1.5, 2.5, 3.5), (-29.0, -48.0, -2.0))
    ext = np.array([v.size[i] * v.voxel[i] for i in range(3)])
    a = rng.uniform(-1, 1, (20000, 3)) * ext
    b = rng.uniform(-1, 1, (20000, 3)) * ext
    b[:3000, 2] = a[:3000, 2]
    b[3000:4000, 1] = a[3000:4000, 1]
    segs = np.concatenate([a, b], axis=1)
    for mode, trunc in ((capi.FIR_GEOMETRY_REFERENCE, True), (capi.FIR_GEOMETRY_EXACT, False)):
        ctx = gpu_ctx_factory()
        ctx.set_option(capi.FIR_OPT_GEOMETRY, mode)
        assert_paths_equal(ctx.siddon_paths(v, segs), restated.siddon_paths(v, segs, truncate=trunc))


def test_setup_divisions_bit_exact_near_parallel_and_wide_range(gpu_ctx_factory, restated):
    """The set-up's quotients come from a correctly rounded reciprocal and two
    fused multiply-add corrections; they must equal the oracle's IEEE
    divisions.  Stress: segments within 1e-5..1e-2 mm of parallel to an axis
    (reciprocals up to 1e5), end points from 1e-3 to 1e3 mm, odd voxel sizes."""
    rng = np.random.default_rng(29)
    v = VolSpec((37, 41, 23), (1.7, 2.3, 3.1), (-30.6, -46.0, -7.0))
    n = 30000
    a = rng.uniform(-1, 1, (n, 3)) * 10.0 ** rng.uniform(-3, 3, (n, 1))
    b = rng.uniform(-1, 1, (n, 3)) * 10.0 ** rng.uniform(-3, 3, (n, 1))
    for k in range(3):
        sl = slice(k * n // 4, (k + 1) * n // 4)
        sign = rng.choice([-1.0, 1.0], sl.stop - sl.start)
        b[sl, k] = a[sl, k] + sign * 10.0 ** rng.uniform(-5, -2, sl.stop - sl.start) * 1.0001
    segs = np.concatenate([a, b], axis=1)
    # non-finite end points, where the quotient falls back to RN(a RN(1/b))
    bad = np.tile(np.array([[-3.0, 2.0, 1.0, 9.0, -7.0, 4.0]]), (18, 1))
    for k, val in enumerate((np.inf, -np.inf, np.nan)):
        for c in range(6):
            bad[k * 6 + c, c] = val
    for mode, trunc in ((capi.FIR_GEOMETRY_REFERENCE, True), (capi.FIR_GEOMETRY_EXACT, False)):
        ctx = gpu_ctx_factory()
        ctx.set_option(capi.FIR_OPT_GEOMETRY, mode)
        assert_paths_equal(ctx.siddon_paths(v, segs), restated.siddon_paths(v, segs, truncate=trunc))
        got = ctx.siddon_paths(v, bad)
        want = restated.siddon_paths(v, bad, truncate=trunc)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


# ------------------------------------------------------------ projectors

def test_forward_tiny_matches_fir_golden(gpu_ctx_factory):
    g = np.load(os.path.join(GOLDEN, "tiny_ref.npz"))
    w = workloads.tiny()
    ctx = gpu_ctx_factory(w.scanner)
    sino = np.zeros(w.n_lors, np.float32)
    ctx.forward(w.vol, g["image"], w.proj, sino)
    np.testing.assert_array_equal(sino, g["sino"])


def test_forward_small_bit_exact_device_and_host(gpu_ctx_factory, restated, torch):
    w = workloads.small()
    x = workloads.activity(w) + np.random.default_rng(3).random(w.vol.shape_zyx, dtype=np.float32)
    want = restated.forward(w.scanner, w.proj, w.vol, x)
    ctx = gpu_ctx_factory(w.scanner)
    host = np.zeros(w.n_lors, np.float32)
    ctx.forward(w.vol, x, w.proj, host)
    np.testing.assert_array_equal(host, want)
    dx = torch.from_numpy(x).cuda()
    dsino = torch.zeros(w.n_lors, dtype=torch.float32, device="cuda")
    ctx.forward(w.vol, dx, w.proj, dsino)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dsino.cpu().numpy(), want)


def test_forward_exact_geometry_non_integer_voxels(gpu_ctx_factory, restated):
    w = workloads.small()
    v = VolSpec.centred((80, 80, 20), (3.2, 3.2, 2.5))
    x = np.random.default_rng(4).random(v.shape_zyx, dtype=np.float32)
    ctx = gpu_ctx_factory(w.scanner)
    ctx.set_option(capi.FIR_OPT_GEOMETRY, capi.FIR_GEOMETRY_EXACT)
    got = np.zeros(w.n_lors, np.float32)
    ctx.forward(v, x, w.proj, got)
    np.testing.assert_array_equal(got, restated.forward(w.scanner, w.proj, v, x, truncate=False))


def test_forward_span3(gpu_ctx_factory, restated):
    s = ScannerSpec.ring(9, 64, 150.0, 4.0)
    p = ProjSpec(9, 64, 5, 0, 3)
    v = VolSpec.centred((48, 48, 18), (4.0, 4.0, 2.0))
    x = np.random.default_rng(8).random(v.shape_zyx, dtype=np.float32)
    ctx = gpu_ctx_factory(s)
    got = np.zeros(capi.proj_geometry(p)["n_bins"], np.float32)
    ctx.forward(v, x, p, got)
    np.testing.assert_array_equal(got, restated.forward(s, p, v, x))


def test_backward_and_sensitivity(gpu_ctx_factory, restated):
    g = np.load(os.path.join(GOLDEN, "tiny_ref.npz"))
    w = workloads.tiny()
    ctx = gpu_ctx_factory(w.scanner)
    bp = np.zeros(4 * w.vol.n_voxels, np.float32)
    ctx.backward(w.proj, g["sino"], w.vol, bp, 4)
    assert_scatter_close(bp.reshape(g["bp4"].shape), g["bp4"])
    sens = np.zeros(4 * w.vol.n_voxels, np.float32)
    ctx.sensitivity(w.proj, w.vol, sens, 4)
    assert_scatter_close(sens.reshape(g["sens4"].shape), g["sens4"])

    w = workloads.small()
    y = np.random.default_rng(9).random(w.n_lors, dtype=np.float32)
    ctx = gpu_ctx_factory(w.scanner)
    for nsub in (1, 4):
        bp = np.zeros(nsub * w.vol.n_voxels, np.float32)
        ctx.backward(w.proj, y, w.vol, bp, nsub)
        assert_scatter_close(bp.reshape(-1, *w.vol.shape_zyx[1:]), restated.backward(w.scanner, w.proj, w.vol, y, nsub))


def test_osem_tiny_and_small(gpu_ctx_factory, restated):
    g = np.load(os.path.join(GOLDEN, "tiny_ref.npz"))
    w = workloads.tiny()
    ctx = gpu_ctx_factory(w.scanner)
    img = np.ones(w.vol.shape_zyx, np.float32)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0])
    ctx.osem(w.proj, g["counts"], w.vol, img, g["sens4"], prm)
    assert rel_l2(img, g["osem"]) <= 1e-4

    w = workloads.small()
    x = workloads.activity(w)
    s = restated.forward(w.scanner, w.proj, w.vol, x)
    y = workloads.poisson_counts(s, w.counts, 7)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    bias = np.full(w.n_lors, 0.02, np.float32)
    prm = OSEMParams(n_iterations=3, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0], cut_radius=120.0)
    want = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    ctx = gpu_ctx_factory(w.scanner)
    img = np.ones_like(x)
    ctx.osem(w.proj, y, w.vol, img, sens, prm, bias=bias)
    assert rel_l2(img, want) <= 1e-4


def test_osem_save_callback_and_subiteration(gpu_ctx_factory, restated, torch):
    w = workloads.tiny()
    g = np.load(os.path.join(GOLDEN, "tiny_ref.npz"))
    ctx = gpu_ctx_factory(w.scanner)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     save_interval=3)
    saved = []
    img = np.ones(w.vol.shape_zyx, np.float32)
    ctx.osem(w.proj, g["counts"], w.vol, img, g["sens4"], prm, save=lambda k, a: saved.append(k))
    assert saved == [3, 6]
    # the same run driven one sub-iteration at a time on device tensors
    d = torch.ones(w.vol.shape_zyx, dtype=torch.float32, device="cuda")
    y = torch.from_numpy(g["counts"]).cuda()
    sens = torch.from_numpy(g["sens4"]).cuda().reshape(4, -1)
    for it in range(2):
        for s in range(4):
            ctx.osem_subiteration(w.proj, y, w.vol, d, sens[s].contiguous(), prm, s, it * 4 + s + 1)
    torch.cuda.synchronize()
    assert rel_l2(d.cpu().numpy(), img) <= 1e-5


# ------------------------------------------------------- image operations

def test_image_and_sinogram_ops_bit_exact(gpu_ctx_factory, restated):
    w = workloads.small()
    rng = np.random.default_rng(12)
    x = (workloads.activity(w) + rng.random(w.vol.shape_zyx, dtype=np.float32)).astype(np.float32)
    ctx = gpu_ctx_factory(w.scanner)
    for fwhm, cut in (([4.0, 4.0, 4.0], 0.0), ([4.0, 4.0, 4.0], 100.0), ([3.0, 5.0, 7.5], 0.0),
                      ([9.0, 2.0, 4.0], 60.0)):
        got = x.copy()
        ctx.convolve(w.vol, got, fwhm, cut)
        np.testing.assert_array_equal(got, restated.convolve(w.vol, x, fwhm, cut))
    for cut in (50.0, 100.0):
        got = x.copy()
        ctx.cut_circle(w.vol, got, cut)
        np.testing.assert_array_equal(got, restated.cut_circle(w.vol, x, cut))
    mask = (rng.random(w.vol.shape_zyx) - 0.3).astype(np.float32)
    got = x.copy()
    ctx.apply_mask(w.vol, got, mask)
    np.testing.assert_array_equal(got, restated.apply_mask(x, mask))
    hu = (rng.random(w.vol.shape_zyx) * 3000 - 1500).astype(np.float32)
    got = hu.copy()
    ctx.hu_to_mu(w.vol, got)
    np.testing.assert_array_equal(got, restated.hu_to_mu(hu))
    bp = (rng.random(w.vol.shape_zyx) * 2).astype(np.float32)
    sens = (rng.random(w.vol.shape_zyx) * 2).astype(np.float32)
    sens[::7] = 0.0
    gi, gb = x.copy(), bp.copy()
    ctx.em_update(w.vol, gi, gb, sens)
    wi, wb = restated.em_update(x, bp, sens)
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gb, wb)
    a = (rng.random(w.n_lors) * 2 - 0.2).astype(np.float32)
    b = (rng.random(w.n_lors) * 2 - 0.2).astype(np.float32)
    got = a.copy()
    ctx.proj_multiply(w.proj, got, b)
    np.testing.assert_array_equal(got, restated.proj_multiply(a, b))
    got = a.copy()
    ctx.proj_exponential(w.proj, got)
    want = restated.exponential(a)
    ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1 and np.mean(ulp == 0) > 0.999


def test_attenuation_factors_fused(gpu_ctx_factory, restated):
    w = workloads.small()
    mu = restated.hu_to_mu(workloads.hounsfield(w))
    want = restated.exponential(restated.forward(w.scanner, w.proj, w.vol, mu))
    ctx = gpu_ctx_factory(w.scanner)
    got = np.zeros(w.n_lors, np.float32)
    ctx.forward_exp(w.vol, mu, w.proj, got)
    ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1 and np.mean(ulp == 0) > 0.999


# ------------------------------------------------------- errors and edges

def test_errors_are_reported_with_fir_messages(gpu_ctx_factory):
    w = workloads.small()
    ctx = gpu_ctx_factory()
    x = np.zeros(w.vol.shape_zyx, np.float32)
    out = np.zeros(w.n_lors, np.float32)
    with pytest.raises(capi.FirError, match="no scanner set"):
        ctx.forward(w.vol, x, w.proj, out)
    ctx.set_scanner(ScannerSpec.ring(8, 64, 200.0, 4.0))
    with pytest.raises(capi.FirError, match=r"Projection must have the same number of rings \(8\) and the same "
                                            r"number of crystals per ring \(64\) as the scanner"):
        ctx.forward(w.vol, x, w.proj, out)
    ctx.set_scanner(w.scanner)
    with pytest.raises(capi.FirError, match="Number of subsets must be a divisor of 64"):
        ctx.backward(w.proj, out, w.vol, np.zeros(3 * w.vol.n_voxels, np.float32), 3)
    with pytest.raises(capi.FirError, match=r"Wrong number of frames \(expected 2\)"):
        capi.lib()  # loaded
        from fir_b200.capi import _check, lib, proj_desc, vol_desc
        import ctypes as C
        _check(lib().fir_backward(ctx.handle, C.byref(proj_desc(w.proj)), out.ctypes.data,
                                  C.byref(vol_desc(w.vol, 1)), x.ctypes.data, 2))
    with pytest.raises(capi.FirError, match="truncates to 0"):
        ctx.forward(VolSpec.centred((8, 8, 8), (0.5, 0.5, 0.5)), np.zeros((8, 8, 8), np.float32), w.proj, out)
    ctx.synchronize()


def test_empty_and_degenerate_inputs(gpu_ctx_factory, restated):
    w = workloads.tiny()
    ctx = gpu_ctx_factory(w.scanner)
    # a volume far outside the scanner: every LOR misses, projections are 0
    v = VolSpec((8, 8, 4), (4.0, 4.0, 4.0), (1000.0, 1000.0, 0.0))
    out = np.full(w.n_lors, 7.0, np.float32)
    ctx.forward(v, np.ones((4, 8, 8), np.float32), w.proj, out)
    assert np.all(out == 0.0)
    bp = np.full(v.n_voxels, 3.0, np.float32)
    ctx.backward(w.proj, np.ones(w.n_lors, np.float32), v, bp, 1)
    assert np.all(bp == 0.0)
    # zero-length path dump requests and zero counts are fine
    r = ctx.siddon_paths(w.vol, np.zeros((0, 6)))
    assert r[0].size == 0
    # non-finite end points end the traversal as FIR's loop does (no hang)
    bad = np.array([[np.nan, 0, 0, 10, 10, 10], [0, 0, 0, np.inf, 1, 1]], np.float64)
    crosses, counts, _, _ = ctx.siddon_paths(w.vol, bad)
    want = restated.siddon_paths(w.vol, bad)
    np.testing.assert_array_equal(crosses, want[0])
    np.testing.assert_array_equal(counts, want[1])


# ---------------------------------------------- full-size properties

def test_clinical_adjoint_and_linearity(gpu_ctx_factory, torch):
    w = workloads.clinical()
    ctx = gpu_ctx_factory(w.scanner)
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(w.vol.shape_zyx, generator=gen, device="cuda")
    y = torch.rand(w.n_lors, generator=gen, device="cuda")
    ax = torch.empty(w.n_lors, device="cuda")
    ctx.forward(w.vol, x, w.proj, ax)
    aty = torch.empty(w.vol.shape_zyx, device="cuda")
    ctx.backward(w.proj, y, w.vol, aty, 1)
    lhs = float(torch.dot(ax.double(), y.double()))
    rhs = float(torch.dot(x.double().ravel(), aty.double().ravel()))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    # scaling by a power of two is exact in every rounding step
    ax2 = torch.empty_like(ax)
    ctx.forward(w.vol, x * 2, w.proj, ax2)
    assert torch.equal(ax2, ax * 2)
    # 16 subsets of the backprojection add up to the full backprojection
    # (float sums in another order: within the 1e-5 projection tolerance)
    sub = torch.empty((16,) + w.vol.shape_zyx, device="cuda")
    ctx.backward(w.proj, y, w.vol, sub, 16)
    torch.cuda.synchronize()
    assert rel_l2(sub.sum(0).cpu().numpy(), aty.cpu().numpy()) <= 1e-5


# ------------------------------------------- resolution-modelling OSEM

def test_osem_psf_matches_oracle(gpu_ctx_factory, restated):
    """fir_osem_psf (Gaussian PSF inside the system model) against the C
    restatement, with bias, cut and the post-filter; with FWHM 0 it is
    fir_osem."""
    w = workloads.small()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 9)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    bias = np.full(w.n_lors, 0.02, np.float32)
    ctx = gpu_ctx_factory(w.scanner)
    for interval, cut in ((0, 0.0), (2, 110.0)):
        prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=interval, fwhm_xyz=[5.0, 5.0, 6.0],
                         cut_radius=cut)
        want = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias, psf=True)
        got = np.ones_like(x)
        ctx.osem(w.proj, y, w.vol, got, sens, prm, bias=bias, psf=True)
        assert rel_l2(got, want) <= 1e-4
        plain = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
        assert rel_l2(want, plain) > 1e-2  # the model differs
    prm0 = OSEMParams(n_iterations=1, n_subsets=4, fwhm_xyz=[0.0, 0.0, 0.0])
    a, b = np.ones_like(x), np.ones_like(x)
    ctx.osem(w.proj, y, w.vol, a, sens, prm0, psf=True)
    ctx.osem(w.proj, y, w.vol, b, sens, prm0)
    assert rel_l2(a, b) <= 1e-5


# ------------------------------------------- bin coordinates, rebin weights

BIN_HEADERS = [
    ProjSpec(8, 128, 15, 43),
    ProjSpec(8, 128, 9, 0),
    ProjSpec(8, 128, 5, 61, 3),
    ProjSpec(8, 96, 3, 0, 5),
    ProjSpec(9, 64, 3, 21, 3),
    ProjSpec(32, 512, 21, 125, 3),
]


def flat_bins(restated, p, coords):
    f = restated.proj(p)
    nax = np.array(f.n_axial[:p.n_segments], np.int64)
    bpv = nax * f.n_tang_coords
    base = np.concatenate([[0], np.cumsum(bpv * f.n_views)])
    si = coords[:, 1] + f.seg_offset
    ok = (coords[:, 0] == 1) & (si >= 0) & (si < p.n_segments)
    si = np.where(ok, si, 0)
    ok &= (coords[:, 2] >= 0) & (coords[:, 2] < f.n_views) & (coords[:, 3] >= 0) & (coords[:, 3] < nax[si])
    flat = base[si] + coords[:, 2] * bpv[si] + coords[:, 3] * f.n_tang_coords + coords[:, 4] + f.tang_offset
    return np.where(ok, flat, -1)


@pytest.mark.parametrize("k", range(len(BIN_HEADERS)))
def test_bin_coordinates_match_oracle(gpu_ctx_factory, restated, k):
    """fir_bin_coordinates equals the restatement of getBinCoordinates (itself
    pinned to compiled FIR) on random crystal pairs, flag and coordinates;
    the flat index is that of the coordinates."""
    p = BIN_HEADERS[k]
    rng = np.random.default_rng(40 + k)
    n = 50000
    pairs = np.stack([rng.integers(0, p.n_rings, n), rng.integers(0, p.n_crystals_per_ring, n),
                      rng.integers(0, p.n_rings, n), rng.integers(0, p.n_crystals_per_ring, n)], axis=1)
    coords, bins = gpu_ctx_factory().bin_coordinates(p, pairs)
    want = restated.bin_coordinates(p, pairs)
    np.testing.assert_array_equal(coords, want)
    np.testing.assert_array_equal(bins, flat_bins(restated, p, want))


def test_bin_coordinates_invert_the_bin_to_crystal_map(gpu_ctx_factory, restated):
    """Span 1, clinical header: the crystal pair of a bin (getCrystalAxialCoord,
    getCrystalAngCoord; rings = slices / 2) maps back to the same bin."""
    p = workloads.clinical().proj
    n = capi.proj_geometry(p)["n_bins"]
    bins = np.sort(np.random.default_rng(3).choice(n, 20000, replace=False))
    t = restated.lor_table_bins(p, bins)
    pairs = np.stack([t[:, 0] // 2, t[:, 1], t[:, 2] // 2, t[:, 3]], axis=1)
    coords, got = gpu_ctx_factory().bin_coordinates(p, pairs)
    assert (coords[:, 0] == 1).all()
    np.testing.assert_array_equal(got, bins)


@pytest.mark.parametrize("k", range(len(BIN_HEADERS)))
def test_rebin_weight_matches_oracle(gpu_ctx_factory, restated, torch, k):
    """fir_proj_rebin_weight equals the restatement bit for bit, on host and
    device buffers (no-op for span 1)."""
    p = BIN_HEADERS[k]
    n = capi.proj_geometry(p)["n_bins"]
    sino = (np.random.default_rng(k).random(n) * 100).astype(np.float32)
    want = restated.rebin_weight(p, sino)
    ctx = gpu_ctx_factory()
    got = sino.copy()
    ctx.proj_rebin_weight(p, got)
    np.testing.assert_array_equal(got, want)
    dev = torch.from_numpy(sino).cuda()
    ctx.proj_rebin_weight(p, dev)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), want)


# ------------------------------------------- ordinary-Poisson (weighted) OSEM

def test_osem_weighted_matches_oracle(gpu_ctx_factory, restated):
    """fir_osem_weighted: measured counts with attenuation factors m = 1 / ACF
    in the model and A_s^T m as sensitivity.  Atomic mode within 1e-4 of the
    restatement, deterministic mode bit-identical to it, and m = 1 gives
    fir_osem."""
    w = workloads.small()
    x = workloads.activity(w)
    mu = restated.hu_to_mu(workloads.hounsfield(w))
    acf = restated.exponential(restated.forward(w.scanner, w.proj, w.vol, mu))
    m = (1.0 / acf).astype(np.float32)
    expect = (restated.forward(w.scanner, w.proj, w.vol, x) * m).astype(np.float32)
    y = workloads.poisson_counts(expect, w.counts, 11)
    sens = restated.backward(w.scanner, w.proj, w.vol.with_frames(4), m, 4)
    bias = np.full(w.n_lors, 0.01, np.float32)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=115.0)
    want = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias, mult=m)
    got = np.ones_like(x)
    gpu_ctx_factory(w.scanner).osem(w.proj, y, w.vol, got, sens, prm, bias=bias, mult=m)
    assert rel_l2(got, want) <= 1e-4
    det = gpu_ctx_factory(w.scanner)
    det.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
    got_det = np.ones_like(x)
    det.osem(w.proj, y, w.vol, got_det, sens, prm, bias=bias, mult=m)
    np.testing.assert_array_equal(got_det, want)
    ones = np.ones_like(m)
    a, b = np.ones_like(x), np.ones_like(x)
    det.osem(w.proj, y, w.vol, a, sens, prm, mult=ones)
    det.osem(w.proj, y, w.vol, b, sens, prm)
    np.testing.assert_array_equal(a, b)


# ------------------------------------------- failure reporting

def test_step_bound_is_reported_and_the_context_recovers(gpu_ctx_factory, restated, torch):
    """A traversal that reaches its step bound sets the device check word; the
    call reports FIR_ERR_DEVICE_CHECK (host buffers at once, device buffers at
    the next synchronize) and the context stays usable.  The bound is forced
    with FIR_OPT_STEP_LIMIT, so no GPU fault is involved.  A bound that no
    path reaches gives FIR's projection bit for bit, which also checks the
    exact tie test against the fast one on every LOR of the workload."""
    w = workloads.small()
    ctx = gpu_ctx_factory(w.scanner)
    x = workloads.activity(w)
    want = restated.forward(w.scanner, w.proj, w.vol, x)
    out = np.zeros(w.n_lors, np.float32)
    ctx.set_option(capi.FIR_OPT_STEP_LIMIT, 3)
    assert ctx.get_option(capi.FIR_OPT_STEP_LIMIT) == 3
    with pytest.raises(capi.FirError, match="iteration bound") as e:
        ctx.forward(w.vol, x, w.proj, out)
    assert e.value.status == 4  # FIR_ERR_DEVICE_CHECK
    dx = torch.from_numpy(x).cuda()
    dout = torch.empty(w.n_lors, device="cuda")
    ctx.forward(w.vol, dx, w.proj, dout)  # enqueued; reported at the synchronize
    with pytest.raises(capi.FirError, match="iteration bound"):
        ctx.synchronize()
    ctx.set_option(capi.FIR_OPT_STEP_LIMIT, 1_000_000)
    ctx.forward(w.vol, x, w.proj, out)
    np.testing.assert_array_equal(out, want)
    ctx.set_option(capi.FIR_OPT_STEP_LIMIT, 0)
    ctx.forward(w.vol, x, w.proj, out)
    np.testing.assert_array_equal(out, want)
    with pytest.raises(capi.FirError, match="must not be negative"):
        ctx.set_option(capi.FIR_OPT_STEP_LIMIT, -1)


def test_osem_from_pinned_host_buffers_is_pipelined_and_identical(gpu_ctx_factory, restated, torch):
    """fir_osem with page-locked host inputs copies them subset by subset on
    a second stream, overlapped with the sub-iterations; with pageable inputs
    they are staged whole.  In deterministic mode both give the same image
    bit for bit (also with bias and multiplicative factors), and the pinned
    inputs are left unchanged."""
    w = workloads.small()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 13)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4).reshape(4, *w.vol.shape_zyx)
    bias = np.full(w.n_lors, 0.02, np.float32)
    m = np.random.default_rng(4).uniform(0.5, 1.0, w.n_lors).astype(np.float32)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=115.0)
    ctx = gpu_ctx_factory(w.scanner)
    ctx.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        return t

    for kw in ({}, {"bias": bias}, {"bias": bias, "mult": m}):
        want = np.ones_like(x)
        ctx.osem(w.proj, y, w.vol, want, sens, prm, **kw)
        py, ps = pinned(y), pinned(sens)
        pkw = {k: pinned(v) for k, v in kw.items()}
        img = pinned(np.ones_like(x))
        ctx.osem(w.proj, py, w.vol, img, ps, prm, **pkw)
        np.testing.assert_array_equal(img.numpy(), want)
        np.testing.assert_array_equal(py.numpy(), y)
        np.testing.assert_array_equal(ps.numpy(), sens)
