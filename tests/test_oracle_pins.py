"""Pins the CPU oracle (oracle/fir_oracle.c) before anything is checked
against it:

1. the golden Siddon paths (generated by FIR itself) reproduce the known
   answers of FIR's unit tests (src_test/SiddonUnitTest.cc:80-423): rows,
   columns and z-lines through every voxel with full-voxel lengths, misses
   along the borders, half-voxel first/last elements for segments starting or
   stopping at a voxel centre;
2. the oracle reproduces every golden path bit for bit, the golden
   ProjGeometry values (src_test/ProjHeaderUnitTest.cc:181-232) and FIR's
   forward/back projection, sensitivity and OSEM of the tiny workload;
3. where the compiled FIR sources are present (oracle/_ref), the oracle is
   bit-identical to FIR on further random and benchmark-geometry cases.
"""
import json
import os

import numpy as np
import pytest

from fir_b200 import workloads
from fir_b200.geometry import OSEMParams, ProjSpec, VolSpec

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _vol(arr):
    return VolSpec(tuple(int(x) for x in arr[0:3]), tuple(arr[3:6]), tuple(arr[6:9]))


@pytest.fixture(scope="module")
def siddon_golden():
    return np.load(os.path.join(GOLDEN, "siddon_cases.npz"))


@pytest.mark.parametrize("name", ["unit3x3x2", "unit512x384"])
def test_golden_paths_are_fir_unit_test_answers(siddon_golden, name):
    g = siddon_golden
    v = _vol(g[name + "_vol"])
    nx, ny, nz = v.size
    vx, vy, vz = v.voxel
    counts, coords, lengths = g[name + "_counts"], g[name + "_coords"], g[name + "_lengths"]
    crosses = g[name + "_crosses"]
    i = 0
    # four misses along the outer lines of slice 0 (SiddonUnitTest.cc:120-153)
    for _ in range(4):
        assert crosses[i] == 0 and counts[i] == 0
        i += 1
    for k in range(nz):
        for j in range(min(ny, 8)):  # rows: SiddonUnitTest.cc:155-197, :345-395
            assert counts[i] == nx
            np.testing.assert_array_equal(coords[i, :nx], k * nx * ny + j * nx + np.arange(nx))
            assert np.all(np.abs(lengths[i, :nx] - vx) < 1e-7)
            i += 1
        for c in range(min(nx, 8)):  # columns: SiddonUnitTest.cc:199-241, :397-423
            assert counts[i] == ny
            np.testing.assert_array_equal(coords[i, :ny], k * nx * ny + c + nx * np.arange(ny))
            assert np.all(np.abs(lengths[i, :ny] - vy) < 1e-7)
            i += 1
    for j in range(min(ny, 4)):  # z-lines: SiddonUnitTest.cc:243-290
        for c in range(min(nx, 4)):
            assert counts[i] == nz
            np.testing.assert_array_equal(coords[i, :nz], c + j * nx + nx * ny * np.arange(nz))
            assert np.all(np.abs(lengths[i, :nz] - vz) < 1e-7)
            i += 1
    # starting at a voxel centre, going backwards (SiddonUnitTest.cc:292-318)
    assert counts[i] == nx // 2 + 1 and coords[i, 0] == nx // 2 and abs(lengths[i, 0] - vx / 2) < 1e-7
    assert counts[i + 1] == ny // 2 + 1 and coords[i + 1, 0] == (ny // 2) * nx and abs(lengths[i + 1, 0] - vy / 2) < 1e-7
    assert coords[i + 2, 0] == (nz - 1) * nx * ny and abs(lengths[i + 2, 0] - vz / 2) < 1e-7
    # stopping at a voxel centre (SiddonUnitTest.cc:320-343)
    last = counts[i + 3] - 1
    assert coords[i + 3, last] == nx // 2 and abs(lengths[i + 3, last] - vx / 2) < 1e-7
    last = counts[i + 4] - 1
    assert coords[i + 4, last] == (ny // 2) * nx and abs(lengths[i + 4, last] - vy / 2) < 1e-7
    last = counts[i + 5] - 1
    assert coords[i + 5, last] == 0 and abs(lengths[i + 5, last] - vz / 2) < 1e-7


@pytest.mark.parametrize("name", ["unit3x3x2", "unit512x384"])
def test_oracle_reproduces_golden_paths(restated, siddon_golden, name):
    g = siddon_golden
    v = _vol(g[name + "_vol"])
    crosses, counts, coords, lengths = restated.siddon_paths(v, g[name + "_segs"])
    np.testing.assert_array_equal(crosses, g[name + "_crosses"])
    np.testing.assert_array_equal(counts, g[name + "_counts"])
    cap = g[name + "_coords"].shape[1]
    for i in range(len(counts)):
        n = counts[i]
        np.testing.assert_array_equal(coords[i, :n], g[name + "_coords"][i, :n])
        np.testing.assert_array_equal(lengths[i, :n], g[name + "_lengths"][i, :n])
    assert cap >= counts.max()


def test_proj_geometry_golden(restated):
    with open(os.path.join(GOLDEN, "proj_geometry.json")) as f:
        geo = json.load(f)
    # literal values of ProjGeometryFillTest (ProjHeaderUnitTest.cc:181-232)
    assert geo["span1_5x32"]["n_bins"] == 1664 and geo["span1_5x32"]["n_axial"] == [4, 5, 4]
    assert geo["span1_5x32"]["max_ring_diff"] == 1 and geo["span1_5x32"]["half_span"] == 0
    assert geo["span3_5x32"]["n_bins"] == 2432 and geo["span3_5x32"]["n_axial"] == [5, 9, 5]
    assert geo["span3_5x32"]["max_ring_diff"] == 4 and geo["span3_5x32"]["half_span"] == 1
    for k, d in geo.items():
        r, c, s, t, span = d["header"]
        f = restated.proj(ProjSpec(r, c, s, t, span))
        assert f.n_bins == d["n_bins"], k
        assert list(f.n_axial[: s]) == d["n_axial"], k
        assert (f.seg_offset, f.tang_offset, f.n_views, f.half_span, f.max_ring_diff) == (
            d["seg_offset"], d["tang_offset"], d["n_views"], d["half_span"], d["max_ring_diff"]), k


def test_oracle_reproduces_tiny_golden(restated):
    g = np.load(os.path.join(GOLDEN, "tiny_ref.npz"))
    w = workloads.tiny()
    np.testing.assert_array_equal(workloads.activity(w), g["image"])
    sino = restated.forward(w.scanner, w.proj, w.vol, g["image"])
    np.testing.assert_array_equal(sino, g["sino"])
    bp4 = restated.backward(w.scanner, w.proj, w.vol, g["sino"], 4)
    np.testing.assert_array_equal(bp4, g["bp4"])
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    np.testing.assert_array_equal(sens, g["sens4"])
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0])
    osem = restated.osem(w.scanner, w.proj, w.vol, g["counts"], np.ones_like(g["image"]), g["sens4"], prm)
    np.testing.assert_array_equal(osem, g["osem"])


# ------------------------------------------------ against compiled FIR

def _clinical_random_lors(w, n, seed):
    rng = np.random.default_rng(seed)
    nb = w.n_lors
    return np.sort(rng.choice(nb, size=n, replace=False)).astype(np.int64)


def test_oracle_bit_identical_to_fir_random_segments(restated, reference):
    rng = np.random.default_rng(11)
    for v in (VolSpec((200, 200, 64), (3.0, 3.0, 3.0), (-298.5, -298.5, 0.0)),
              VolSpec((33, 17, 9), (2.0, 3.0, 5.0), (-30.0, -20.0, 4.0)),
              VolSpec((40, 40, 20), (1.5, 2.5, 3.5), (-29.0, -48.0, -2.0))):
        ext = np.array([v.size[i] * v.voxel[i] for i in range(3)])
        a = rng.uniform(-1, 1, (3000, 3)) * ext
        b = rng.uniform(-1, 1, (3000, 3)) * ext
        b[:500, 2] = a[:500, 2]
        b[500:700, 0] = a[500:700, 0]
        segs = np.concatenate([a, b], axis=1)
        r1 = restated.siddon_paths(v, segs, truncate=True)
        r2 = reference.siddon_paths(v, segs)
        for x, y in zip(r1, r2):
            np.testing.assert_array_equal(x, y)


def test_oracle_bit_identical_to_fir_small_workload(restated, reference):
    w = workloads.small()
    reference.threads(1)
    x = workloads.activity(w)
    nb = w.n_lors
    s1 = restated.forward(w.scanner, w.proj, w.vol, x)
    s2 = reference.forward(w.scanner, w.proj, w.vol, x, nb)
    np.testing.assert_array_equal(s1, s2)
    hu = workloads.hounsfield(w)
    np.testing.assert_array_equal(restated.hu_to_mu(hu), reference.hu_to_mu(w.vol, hu))
    mu = restated.hu_to_mu(hu)
    acf = restated.exponential(restated.forward(w.scanner, w.proj, w.vol, mu))
    acf_ref = reference.exponential(w.proj, reference.forward(w.scanner, w.proj, w.vol, mu, nb))
    np.testing.assert_array_equal(acf, acf_ref)
    np.testing.assert_array_equal(restated.proj_multiply(s1, acf), reference.proj_multiply(w.proj, s2, acf_ref))
    for cut in (0.0, 100.0):
        np.testing.assert_array_equal(restated.convolve(w.vol, x, [4.0, 4.0, 4.0], cut),
                                      reference.convolve(w.vol, x, [4.0, 4.0, 4.0], cut))
        np.testing.assert_array_equal(restated.cut_circle(w.vol, x, cut), reference.cut_circle(w.vol, x, cut))
    np.testing.assert_array_equal(restated.convolve(w.vol, x, [3.0, 5.0, 7.5], 0.0),
                                  reference.convolve(w.vol, x, [3.0, 5.0, 7.5], 0.0))
    mask = (np.random.default_rng(1).random(x.shape) - 0.3).astype(np.float32)
    np.testing.assert_array_equal(restated.apply_mask(x, mask), reference.apply_mask(w.vol, x, mask))
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    np.testing.assert_array_equal(sens, reference.sensitivity(w.scanner, w.proj, w.vol.with_frames(4), 4))
    bias = np.full(nb, 0.05, np.float32)
    prm = OSEMParams(n_iterations=1, n_subsets=4, convolution_interval=2, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=110.0)
    y = workloads.poisson_counts(s1, w.counts, 3)
    o1 = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    o2 = reference.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    np.testing.assert_array_equal(o1, o2)


@pytest.mark.parametrize("extra_frames,cut,interval", [(1, 110.0, 2), (0, 0.0, 1)])
def test_oracle_reso_reco_bit_identical_to_fir(restated, reference, extra_frames, cut, interval):
    """OSEM_ResoReco as FIR runs it (reconAlgos.cc:203-367): the restatement
    against FIR's own function on one thread, image and sensitivity (every
    frame of which FIR filters in place) bit for bit."""
    w = workloads.small()
    reference.threads(1)
    x = workloads.activity(w)
    nb = reference.proj_geometry(w.proj)["n_bins"]
    s1 = restated.forward(w.scanner, w.proj, w.vol, x)
    y = workloads.poisson_counts(s1, w.counts, 4)
    sens4 = restated.sensitivity(w.scanner, w.proj, w.vol, 4).reshape(4, -1)
    sens = np.concatenate([sens4] + [sens4.sum(axis=0, keepdims=True)] * extra_frames)
    bias = np.full(nb, 0.02, np.float32)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=interval, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=cut)
    i1, sn1 = restated.osem_reso_reco(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    i2, sn2 = reference.osem_reso_reco(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, bias=bias)
    np.testing.assert_array_equal(sn1, sn2)
    np.testing.assert_array_equal(i1, i2)
    assert not np.array_equal(sn1, sens.ravel()) and float(i1.max()) > 0


def test_oracle_span3_and_lor_tables(restated, reference):
    for p in (ProjSpec(5, 32, 3, 8, 3), ProjSpec(9, 64, 5, 0, 3), ProjSpec(8, 128, 15, 43, 1)):
        nb = reference.proj_geometry(p)["n_bins"]
        np.testing.assert_array_equal(restated.lor_table(p), reference.lor_table(p, nb))


def test_oracle_psf_osem_reduces_to_osem_without_psf(restated):
    """The resolution-modelling OSEM of the restatement with FWHM 0 is
    bit-identical to its OSEM, and with a PSF it differs."""
    from fir_b200 import workloads
    from fir_b200.geometry import OSEMParams

    w = workloads.tiny()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 1)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    prm0 = OSEMParams(n_iterations=1, n_subsets=4, fwhm_xyz=[0.0, 0.0, 0.0])
    a = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm0)
    b = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm0, psf=True)
    np.testing.assert_array_equal(a, b)
    prm = OSEMParams(n_iterations=1, n_subsets=4, fwhm_xyz=[4.0, 4.0, 4.0])
    c = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, psf=True)
    assert np.abs(c - a).max() > 1e-3


BIN_HEADERS = [
    ProjSpec(8, 128, 15, 43),          # span 1, all ring differences, FOV-limited
    ProjSpec(8, 128, 9, 0),            # span 1, 9 of 15 segments, all tangential bins
    ProjSpec(8, 128, 5, 61, 3),        # span 3
    ProjSpec(8, 96, 3, 0, 5),          # span 5
    ProjSpec(9, 64, 3, 21, 3),         # span 3, odd ring count, max ring difference 4
]


def random_pairs(p, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, p.n_rings, n), rng.integers(0, p.n_crystals_per_ring, n),
                     rng.integers(0, p.n_rings, n), rng.integers(0, p.n_crystals_per_ring, n)], axis=1)


@pytest.mark.parametrize("k", range(len(BIN_HEADERS)))
def test_bin_coordinates_pinned_to_fir(restated, reference, k):
    """ProjData::getBinCoordinates: the restatement equals compiled FIR on
    random crystal pairs (flag and all four coordinates)."""
    p = BIN_HEADERS[k]
    pairs = random_pairs(p, 20000, k)
    got = restated.bin_coordinates(p, pairs)
    want = reference.bin_coordinates(p, pairs)
    np.testing.assert_array_equal(got, want)
    assert got[:, 0].sum() > 1000


# FIR's ProjData::getInd adds the segment offset twice (ProjData.inl:76-79
# with ProjHeader.inl:55), so its bin accessors, and rebinWeight through them,
# index the wrong row once a sinogram has more than one segment (a heap
# overflow under AddressSanitizer).  FIR's own rebinWeight is therefore
# compared only where that offset is 0 (one segment); elsewhere the
# restatement is checked against an independent count of ring pairs.
REBIN_FIR_VALID = [ProjSpec(8, 128, 15, 43), ProjSpec(8, 128, 1, 61, 3), ProjSpec(8, 96, 1, 0, 5),
                   ProjSpec(9, 64, 1, 21, 3)]


@pytest.mark.parametrize("k", range(len(REBIN_FIR_VALID)))
def test_rebin_weight_pinned_to_fir(restated, reference, k):
    """ProjData::rebinWeight, single-segment headers: bit-identical to
    compiled FIR (a no-op for span 1)."""
    p = REBIN_FIR_VALID[k]
    n = restated.proj(p).n_bins
    sino = (np.random.default_rng(k).random(n) * 10).astype(np.float32)
    got = restated.rebin_weight(p, sino)
    np.testing.assert_array_equal(got, reference.rebin_weight(p, sino))
    if p.segment_span > 1:
        assert (got != sino).any()
    else:
        np.testing.assert_array_equal(got, sino)


def rebin_factors_by_counting(restated, p):
    """Per (segment, axial): the number w of ring pairs (r1, r2) that a span-s
    sinogram merges into it, counted directly from the segment and axial
    coordinate of each pair (getBinCoordinates' axial mapping); the bin
    factor is (float)(1 / w) where w > 1, else 1."""
    f = restated.proj(p)
    half, span = f.half_span, p.segment_span
    count = {}
    for r1 in range(p.n_rings):
        for r2 in range(p.n_rings):
            d = r1 - r2
            a = abs(d)
            if a > f.max_ring_diff:
                continue
            if a <= half:
                seg, m = 0, 0
            else:
                k = 1 + (a - half - 1) // span
                seg, m = (k if d > 0 else -k), 1 + half + (k - 1) * span
            key = (seg, r1 + r2 - m)
            count[key] = count.get(key, 0) + 1
    return {k: (np.float32(1.0 / v) if v > 1 else np.float32(1.0)) for k, v in count.items()}


@pytest.mark.parametrize("k", [2, 3, 4])
def test_rebin_weight_multi_segment_by_counting(restated, k):
    p = BIN_HEADERS[k]
    f = restated.proj(p)
    ones = np.ones(f.n_bins, np.float32)
    got = restated.rebin_weight(p, ones)
    want = np.ones_like(ones)
    fac = rebin_factors_by_counting(restated, p)
    base = 0
    for si in range(p.n_segments):
        seg = si - f.seg_offset
        nax = f.n_axial[si]
        block = want[base:base + f.n_views * nax * f.n_tang_coords].reshape(f.n_views, nax, f.n_tang_coords)
        for ax in range(nax):
            block[:, ax, :] = fac.get((seg, ax), np.float32(1.0))
        base += f.n_views * nax * f.n_tang_coords
    np.testing.assert_array_equal(got, want)
    assert (got < 1).any()


def test_oracle_weighted_osem_with_unit_factors_is_osem(restated):
    """The ordinary-Poisson OSEM of the restatement with m = 1 is
    bit-identical to its OSEM."""
    from fir_b200 import workloads
    from fir_b200.geometry import OSEMParams

    w = workloads.tiny()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 1)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, 4)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0])
    a = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm)
    b = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm, mult=np.ones_like(y))
    np.testing.assert_array_equal(a, b)
