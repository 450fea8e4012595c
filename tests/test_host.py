"""CPU tests of the native boundary: the C-ABI library loads and exports
every entry point include/fir_cuda.h declares; its host helpers (header
validation, ProjGeometry, scanner tables) agree with the oracle and with
FIR's messages; Interfile files round-trip.  No GPU call is made."""
import os
import re

import numpy as np
import pytest

from fir_b200 import capi, interfile, workloads
from fir_b200.geometry import ProjSpec, ScannerSpec, VolSpec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "fir_cuda.h")).read()
    return sorted(set(re.findall(r"^\s*(?:fir_status|int|const char\*|long long)\s+(fir_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(capi.exported_symbols())
    assert L.fir_abi_version() == 1


def test_no_device_is_reported_not_faked():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(capi.FirError) as e:
        capi.Context()
    assert e.value.name == "FIR_ERR_NO_DEVICE"


@pytest.mark.parametrize("case", [
    # ProjHeaderCheckTest (src_test/ProjHeaderUnitTest.cc:23-175)
    (ProjSpec(0, 4), '"number of rings" must be provided and > 0'),
    (ProjSpec(-1, 4), '"number of rings" must be provided and > 0'),
    (ProjSpec(1, 0), '"number of crystals per ring" must be provided and > 0'),
    (ProjSpec(1, -1), '"number of crystals per ring" must be provided and > 0'),
    (ProjSpec(1, 3), '"number of crystals per ring" must be a multiple of four'),
    (ProjSpec(2, 4, 1, 0, 0), '"segment span" must be > 0'),
    (ProjSpec(2, 4, 1, 0, -1), '"segment span" must be > 0'),
    (ProjSpec(2, 4, 1, 0, 2), '"segment span" must be an odd number'),
    (ProjSpec(2, 4, 1, 0, 5), 'For 2 ring(s), "segment span" must not be > 3'),
    (ProjSpec(2, 4, 0), '"number of segments" must be an odd number'),
    (ProjSpec(2, 4, -1), '"number of segments" must not be negative'),
    (ProjSpec(2, 4, 2), '"number of segments" must be an odd number'),
    (ProjSpec(2, 4, 5), 'For 2 ring(s) and a segment span of 1, "number of segments" must not be > 3'),
    (ProjSpec(2, 4, 1, -1), '"number of tangential coordinates" must not be negative'),
    (ProjSpec(2, 4, 1, 4), 'For 4 crystals per ring, "number of tangential coordinates" must not be > 3'),
])
def test_proj_header_validation_messages(case):
    spec, msg = case
    with pytest.raises(capi.FirError) as e:
        capi.proj_geometry(spec)
    assert msg in str(e.value)
    assert e.value.name == "FIR_ERR_INVALID_ARGUMENT"


def test_proj_header_valid_cases_and_default_tang():
    assert capi.proj_geometry(ProjSpec(1, 4))["n_bins"] > 0
    assert capi.proj_geometry(ProjSpec(2, 4, 1, 0, 3))["n_bins"] > 0
    assert capi.proj_geometry(ProjSpec(2, 4, 3))["n_bins"] > 0
    assert capi.proj_geometry(ProjSpec(2, 4, 1, 0))["n_tang_coords"] == 3


@pytest.mark.parametrize("p", [ProjSpec(5, 32, 3, 8, 1), ProjSpec(5, 32, 3, 8, 3), ProjSpec(39, 624, 3, 380, 3),
                               ProjSpec(32, 512, 63, 125), ProjSpec(64, 640, 127, 163), ProjSpec(24, 96, 15, 0, 3)])
def test_proj_geometry_matches_oracle(restated, p):
    g = capi.proj_geometry(p)
    f = restated.proj(p)
    assert g["n_bins"] == f.n_bins
    assert g["n_axial"] == list(f.n_axial[: p.n_segments])
    assert (g["seg_offset"], g["tang_offset"], g["n_views"], g["half_span"], g["max_ring_diff"]) == (
        f.seg_offset, f.tang_offset, f.n_views, f.half_span, f.max_ring_diff)


@pytest.mark.parametrize("s", [
    ScannerSpec.ring(8, 128, 200.0, 4.0),
    ScannerSpec.ring(32, 512, 400.0, 4.0),
    ScannerSpec.ring(64, 640, 410.0, 3.2),
    # modular scanner: 8x8 crystal blocks, 4x1 modules per rSector, gaps
    ScannerSpec(rsector_repeat_number=24, rsector_inner_radius=350.0, crystal_dims=(20.0, 4.0, 4.2),
                crystal_repeat=(8, 8), inter_crystal=(0.1, 0.2), module_repeat=(2, 3), inter_module=(0.5, 1.0)),
    ScannerSpec(rsector_repeat_number=7, rsector_inner_radius=100.0, crystal_dims=(10.0, 3.0, 3.0),
                crystal_repeat=(5, 2), rsector_dims=(12.0, 0.0, 0.0)),
])
def test_scanner_tables_match_oracle(restated, s):
    xy, z = capi.scanner_tables(s)
    xy2, z2 = restated.scanner_tables(s)
    np.testing.assert_array_equal(xy.ravel(), xy2)
    np.testing.assert_array_equal(z, z2)


def test_scanner_validation():
    bad = ScannerSpec(rsector_repeat_number=0, rsector_inner_radius=100.0)
    with pytest.raises(capi.FirError, match='"rSector repeat number" must be present and > 0'):
        capi.scanner_tables(bad)
    bad = ScannerSpec(rsector_repeat_number=8, rsector_inner_radius=100.0, crystal_repeat=(2, 1))
    with pytest.raises(capi.FirError, match="Crystal repeat number in Y cannot be > 1"):
        capi.scanner_tables(bad)
    bad = ScannerSpec(rsector_repeat_number=8, rsector_inner_radius=100.0, crystal_dims=(5.0, 2.0, 2.0),
                      module_dims=(4.0, 0.0, 0.0))
    with pytest.raises(capi.FirError, match="Module dimension in X must be >= 5"):
        capi.scanner_tables(bad)


def test_interfile_roundtrips(tmp_path):
    w = workloads.small()
    s_path = str(tmp_path / "scanner.scan")
    interfile.write_scanner(s_path, w.scanner)
    s2 = interfile.read_scanner(s_path)
    np.testing.assert_array_equal(capi.scanner_tables(s2)[0], capi.scanner_tables(w.scanner)[0])
    nb = capi.proj_geometry(w.proj)["n_bins"]
    data = np.random.default_rng(0).random(nb, dtype=np.float32)
    hs = interfile.write_proj(str(tmp_path / "sino"), w.proj, data)
    p2, arr = interfile.read_proj(hs, nb)
    assert p2 == w.proj
    np.testing.assert_array_equal(arr, data)
    img = workloads.activity(w)
    h = interfile.write_vol(str(tmp_path / "img"), w.vol, img)
    v2, arr2 = interfile.read_vol(h)
    assert tuple(v2.size) == tuple(w.vol.size)
    np.testing.assert_array_equal(arr2, img)


def test_interfile_keyword_rules_and_formats(tmp_path):
    os.environ["FIR_TEST_DIR"] = str(tmp_path)
    raw = (np.arange(24) - 5).astype(">i2")
    raw.tofile(tmp_path / "v.i33")
    hdr = tmp_path / "v.h33"
    hdr.write_text(
        "  !INTERFILE  :=\n"
        "NAME_OF_DATA_FILE := ${FIR_TEST_DIR}/v.i33\n"
        "number format := signed integer\n"
        "!number of bytes per pixel := 2\n"
        "imagedata byte order := BIGENDIAN\n"
        "matrix size[1] := 4\nMATRIX SIZE [2] := 3\nnumber of slices := 2\n"
        "scaling factor (mm/pixel) [1] := 1.5\nscaling factor (mm/pixel) [2] := 2\nslice thickness (pixels) := 3\n"
        "!END OF INTERFILE :=\n")
    v, d = interfile.read_vol(str(hdr))
    assert tuple(v.size) == (4, 3, 2) and tuple(v.voxel) == (1.5, 2.0, 3.0)
    np.testing.assert_array_equal(d.ravel(), np.arange(24) - 5)
