"""Test infrastructure only: ctypes bindings of the two CPU oracles.

* :class:`Restated` -- ``oracle/libfir_oracle.so``, our C restatement of FIR's
  algorithms (fir_oracle.c).  Always available once ``make -C oracle restated``
  ran.
* :class:`Reference` -- ``oracle/_ref/libfirref.so``, FIR's own sources compiled
  with the harness ``ref_harness.cc``.  Available where it was built from a FIR
  checkout; it is copied as a built file to machines without the sources.

Arrays are numpy; sinograms are flat float32 in FIR's file order, volumes are
float32 ``[frames*nz, ny, nx]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

from fir_b200.geometry import ProjSpec, ScannerSpec, VolSpec, OSEMParams
from fir_b200 import interfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
RESTATED_SO = os.path.join(HERE, "libfir_oracle.so")
REF_BIN = os.path.join(HERE, "_ref")
DROPIN_BIN = os.path.join(HERE, "_ref", "dropin")
REF_SO = os.path.join(HERE, "_ref", "libfirref.so")
# FIR checkout whose sources build the reference oracle; the build is
# skipped, with a message, when it is not given.
REF_SOURCES = os.environ.get("FIR_REFERENCE_SRC", "")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build(reference: bool = True, source: Optional[str] = None) -> None:
    """Builds the restatement, and the reference (plus FIR's executables
    compiled against the drop-in layer) from the FIR checkout ``source``
    (default: $FIR_REFERENCE_SRC).  Without a checkout only the restatement
    is built; the reference oracle is then whatever oracle/_ref holds."""
    targets = ["restated"]
    src = source or REF_SOURCES
    if reference and src and os.path.isdir(os.path.join(src, "src_lib")):
        targets.append("reference")
        if os.path.exists(os.path.join(ROOT, "fir_b200", "lib", "libfir.so")):
            targets.append("dropin")
    elif reference:
        print("oracle: no FIR checkout given (FIR_REFERENCE_SRC); the reference oracle is not rebuilt")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={src}", "-j8"] + targets, check=True)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


# ------------------------------------------------------------- restatement

class FoVol(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("vx", C.c_double), ("vy", C.c_double), ("vz", C.c_double),
        ("ox", C.c_double), ("oy", C.c_double), ("oz", C.c_double),
    ]


class FoProj(C.Structure):
    _fields_ = [
        ("n_rings", C.c_int), ("n_crystals_per_ring", C.c_int), ("segment_span", C.c_int),
        ("n_segments", C.c_int), ("n_tang_coords", C.c_int),
        ("n_bins", C.c_longlong),
        ("seg_offset", C.c_int), ("tang_offset", C.c_int), ("n_views", C.c_int),
        ("half_span", C.c_int), ("max_ring_diff", C.c_int),
        ("n_axial", C.c_int * 1024),
    ]


class FoScanner(C.Structure):
    _fields_ = [
        ("crystal_dims", C.c_double * 3), ("crystal_repeat", C.c_int * 2),
        ("inter_crystal", C.c_double * 2), ("module_dims", C.c_double * 3),
        ("module_repeat", C.c_int * 2), ("inter_module", C.c_double * 2),
        ("rsector_dims", C.c_double * 3), ("rsector_repeat", C.c_int),
        ("rsector_inner_radius", C.c_double),
    ]


class FoGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("ext", C.c_double * 3), ("low", C.c_double * 3), ("high", C.c_double * 3),
    ]


class FoOsem(C.Structure):
    _fields_ = [
        ("n_iterations", C.c_int), ("n_subsets", C.c_int), ("convolution_interval", C.c_int),
        ("cut_radius", C.c_float), ("fwhm", C.c_float * 3),
    ]


def fo_vol(v: VolSpec) -> FoVol:
    return FoVol(int(v.size[0]), int(v.size[1]), int(v.size[2]),
                 float(v.voxel[0]), float(v.voxel[1]), float(v.voxel[2]),
                 float(v.offset[0]), float(v.offset[1]), float(v.offset[2]))


def fo_scanner(s: ScannerSpec) -> FoScanner:
    f = FoScanner()
    f.crystal_dims[:] = [float(x) for x in s.crystal_dims]
    f.crystal_repeat[:] = [int(x) for x in s.crystal_repeat]
    f.inter_crystal[:] = [float(x) for x in s.inter_crystal]
    f.module_dims[:] = [float(x) for x in s.module_dims]
    f.module_repeat[:] = [int(x) for x in s.module_repeat]
    f.inter_module[:] = [float(x) for x in s.inter_module]
    f.rsector_dims[:] = [float(x) for x in s.rsector_dims]
    f.rsector_repeat = int(s.rsector_repeat_number)
    f.rsector_inner_radius = float(s.rsector_inner_radius)
    return f


class Restated:
    """The C restatement of FIR's algorithm (serial, FIR's loop order)."""

    def __init__(self, path: str = RESTATED_SO):
        if not os.path.exists(path):
            build(reference=False)
        L = C.CDLL(path)
        self.L = L
        L.fo_proj_fill.argtypes = [C.POINTER(FoProj)]
        L.fo_scanner_tables.argtypes = [C.POINTER(FoScanner), _f64p, _f64p]
        L.fo_grid_init.argtypes = [C.POINTER(FoGrid), C.POINTER(FoVol), C.c_int]
        L.fo_siddon.argtypes = [C.POINTER(FoGrid)] + [C.c_double] * 6 + [
            _i32p, _f64p, C.c_int, C.POINTER(C.c_int)]
        L.fo_forward.argtypes = [C.POINTER(FoVol), C.c_int, _f32p, C.POINTER(FoProj), _f64p, _f64p, _f32p]
        L.fo_backward.argtypes = [C.POINTER(FoProj), C.c_void_p, C.POINTER(FoVol), C.c_int, _f64p, _f64p,
                                  C.c_int, _f32p]
        L.fo_osem.argtypes = [C.POINTER(FoProj), _f32p, C.c_void_p, C.POINTER(FoVol), C.c_int, _f64p, _f64p,
                              _f32p, _f32p, C.POINTER(FoOsem)]
        L.fo_osem_psf.argtypes = L.fo_osem.argtypes
        L.fo_precision_study.argtypes = [C.POINTER(FoProj), _f64p, _f64p, C.POINTER(FoVol), C.c_int, _f32p,
                                         np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS"), C.c_longlong,
                                         C.c_int, _f64p]
        L.fo_osem_reso_reco.argtypes = [C.POINTER(FoProj), _f32p, C.c_void_p, C.POINTER(FoVol), C.c_int, _f64p,
                                        _f64p, _f32p, _f32p, C.c_int, C.POINTER(FoOsem)]
        L.fo_osem_weighted.argtypes = [C.POINTER(FoProj), _f32p, _f32p, C.c_void_p, C.POINTER(FoVol), C.c_int,
                                       _f64p, _f64p, _f32p, _f32p, C.POINTER(FoOsem)]
        L.fo_bin_coordinates.argtypes = [C.POINTER(FoProj)] + [C.c_int] * 4 + [C.POINTER(C.c_int)] * 4
        L.fo_rebin_weight.argtypes = [C.POINTER(FoProj), _f32p]
        L.fo_em_update.argtypes = [C.c_longlong, _f32p, _f32p, _f32p]
        L.fo_convolve.argtypes = [C.POINTER(FoVol), _f32p, _f32p, C.c_float]
        L.fo_cut_circle.argtypes = [C.POINTER(FoVol), _f32p, C.c_float]
        L.fo_apply_mask.argtypes = [C.c_longlong, _f32p, _f32p]
        L.fo_hu_to_mu.argtypes = [C.c_longlong, _f32p]
        L.fo_exponential.argtypes = [C.c_longlong, _f32p]
        L.fo_proj_multiply.argtypes = [C.c_longlong, _f32p, _f32p]
        L.fo_crystal_axial.argtypes = [C.POINTER(FoProj), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.fo_crystal_ang.argtypes = [C.POINTER(FoProj), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]

    def proj(self, p: ProjSpec) -> FoProj:
        f = FoProj(p.n_rings, p.n_crystals_per_ring, p.segment_span, p.n_segments, p.n_tang_coords)
        rc = self.L.fo_proj_fill(C.byref(f))
        if rc != 0:
            raise ValueError(f"invalid projection header (code {rc})")
        return f

    def scanner_tables(self, s: ScannerSpec):
        xy = np.zeros(2 * s.n_crystals_per_ring, np.float64)
        z = np.zeros(2 * s.n_rings - 1, np.float64)
        if self.L.fo_scanner_tables(C.byref(fo_scanner(s)), xy, z) != 0:
            raise ValueError("invalid scanner header")
        return xy, z

    def lor_table(self, p: ProjSpec) -> np.ndarray:
        f = self.proj(p)
        out = np.zeros((f.n_bins, 4), np.int32)
        a1, a2, c1, c2 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        b = 0
        for seg in range(-f.seg_offset, f.seg_offset + 1):
            for view in range(f.n_views):
                for ax in range(f.n_axial[seg + f.seg_offset]):
                    self.L.fo_crystal_axial(C.byref(f), seg, ax, C.byref(a1), C.byref(a2))
                    for t in range(-f.tang_offset, -f.tang_offset + f.n_tang_coords):
                        self.L.fo_crystal_ang(C.byref(f), view, t, C.byref(c1), C.byref(c2))
                        out[b] = (a1.value, c1.value, a2.value, c2.value)
                        b += 1
        return out

    def lor_table_bins(self, p: ProjSpec, bins) -> np.ndarray:
        """Crystal pairs (axial1, ang1, axial2, ang2) of the given flat bins."""
        f = self.proj(p)
        bins = np.asarray(bins, np.int64).ravel()
        nax = np.array(f.n_axial[: p.n_segments], np.int64)
        bpv = nax * f.n_tang_coords
        base = np.concatenate([[0], np.cumsum(bpv * f.n_views)])
        k = np.searchsorted(base, bins, side="right") - 1
        r = bins - base[k]
        view = r // bpv[k]
        rem = r - view * bpv[k]
        axial = rem // f.n_tang_coords
        tang = rem - axial * f.n_tang_coords - f.tang_offset
        seg = k - f.seg_offset
        out = np.zeros((bins.size, 4), np.int32)
        a1, a2, c1, c2 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        for i in range(bins.size):
            self.L.fo_crystal_axial(C.byref(f), int(seg[i]), int(axial[i]), C.byref(a1), C.byref(a2))
            self.L.fo_crystal_ang(C.byref(f), int(view[i]), int(tang[i]), C.byref(c1), C.byref(c2))
            out[i] = (a1.value, c1.value, a2.value, c2.value)
        return out

    def siddon_paths(self, v: VolSpec, pts: np.ndarray, truncate: bool = True):
        """Per-segment paths: returns (crosses[n], counts[n], coords[n,cap], lengths[n,cap])."""
        g = FoGrid()
        self.L.fo_grid_init(C.byref(g), C.byref(fo_vol(v)), int(truncate))
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 6)
        n = pts.shape[0]
        cap = int(v.size[0] + v.size[1] + v.size[2] + 2)
        coords = np.full((n, cap), -1, np.int32)
        lengths = np.zeros((n, cap), np.float64)
        crosses = np.zeros(n, np.int32)
        counts = np.zeros(n, np.int32)
        cnt = C.c_int()
        for i in range(n):
            crosses[i] = self.L.fo_siddon(C.byref(g), *[float(x) for x in pts[i]], coords[i], lengths[i], cap,
                                          C.byref(cnt))
            counts[i] = cnt.value
        return crosses, counts, coords, lengths

    def forward(self, s: ScannerSpec, p: ProjSpec, v: VolSpec, img: np.ndarray, truncate: bool = True):
        f = self.proj(p)
        xy, z = self.scanner_tables(s)
        out = np.zeros(f.n_bins, np.float32)
        self.L.fo_forward(C.byref(fo_vol(v)), int(truncate), np.ascontiguousarray(img, np.float32).ravel(),
                          C.byref(f), xy, z, out)
        return out

    def backward(self, s: ScannerSpec, p: ProjSpec, v: VolSpec, sino: Optional[np.ndarray], n_subsets: int = 1,
                 truncate: bool = True):
        f = self.proj(p)
        xy, z = self.scanner_tables(s)
        out = np.zeros(v.n_voxels * n_subsets, np.float32)
        sino_arr = None if sino is None else np.ascontiguousarray(sino, np.float32)
        ptr = None if sino_arr is None else sino_arr.ctypes.data_as(C.c_void_p)
        self.L.fo_backward(C.byref(f), ptr, C.byref(fo_vol(v)), int(truncate), xy, z, n_subsets, out)
        return out.reshape(n_subsets * v.size[2], v.size[1], v.size[0])

    def sensitivity(self, s, p, v, n_subsets: int = 1, truncate: bool = True):
        return self.backward(s, p, v, None, n_subsets, truncate)

    def osem(self, s, p, v, sino, img, sens, prm: OSEMParams, bias=None, truncate: bool = True, psf: bool = False,
             mult=None):
        """reconAlgos::OSEM; with psf, the corrected resolution-modelling OSEM;
        with mult, the ordinary-Poisson model with multiplicative factors."""
        f = self.proj(p)
        xy, z = self.scanner_tables(s)
        img = np.ascontiguousarray(img, np.float32).copy().ravel()
        o = FoOsem(prm.n_iterations, prm.n_subsets, prm.convolution_interval, prm.cut_radius)
        o.fwhm[:] = [float(x) for x in prm.fwhm_xyz]
        bias_arr = None if bias is None else np.ascontiguousarray(bias, np.float32)
        bptr = None if bias_arr is None else bias_arr.ctypes.data_as(C.c_void_p)
        if mult is not None:
            self.L.fo_osem_weighted(C.byref(f), np.ascontiguousarray(sino, np.float32),
                                    np.ascontiguousarray(mult, np.float32), bptr, C.byref(fo_vol(v)), int(truncate),
                                    xy, z, img, np.ascontiguousarray(sens, np.float32).ravel(), C.byref(o))
            return img.reshape(v.shape_zyx)
        fn = self.L.fo_osem_psf if psf else self.L.fo_osem
        fn(C.byref(f), np.ascontiguousarray(sino, np.float32), bptr, C.byref(fo_vol(v)), int(truncate), xy, z, img,
           np.ascontiguousarray(sens, np.float32).ravel(), C.byref(o))
        return img.reshape(v.shape_zyx)

    def osem_reso_reco(self, s, p, v, sino, img, sens, prm: OSEMParams, bias=None, truncate: bool = True):
        """reconAlgos::OSEM_ResoReco as FIR runs it; returns (image, sens),
        every frame of sens filtered in place."""
        f = self.proj(p)
        xy, z = self.scanner_tables(s)
        img = np.ascontiguousarray(img, np.float32).copy().ravel()
        sens = np.ascontiguousarray(sens, np.float32).copy().ravel()
        o = FoOsem(prm.n_iterations, prm.n_subsets, prm.convolution_interval, prm.cut_radius)
        o.fwhm[:] = [float(x) for x in prm.fwhm_xyz]
        bias_arr = None if bias is None else np.ascontiguousarray(bias, np.float32)
        bptr = None if bias_arr is None else bias_arr.ctypes.data_as(C.c_void_p)
        self.L.fo_osem_reso_reco(C.byref(f), np.ascontiguousarray(sino, np.float32), bptr, C.byref(fo_vol(v)),
                                 int(truncate), xy, z, img, sens, sens.size // v.n_voxels, C.byref(o))
        return img.reshape(v.shape_zyx), sens

    def precision_study(self, s, p, v, img, bins, precision: int, truncate: bool = True) -> dict:
        """FIR's double traversal against a float one (precision 1: double
        set-up, float loop; 2: float set-up and loop) over the given bins."""
        f = self.proj(p)
        xy, z = self.scanner_tables(s)
        out = np.zeros(5, np.float64)
        b = np.ascontiguousarray(bins, np.int64)
        self.L.fo_precision_study(C.byref(f), xy, z, C.byref(fo_vol(v)), int(truncate),
                                  np.ascontiguousarray(img, np.float32).ravel(), b, b.size, int(precision), out)
        return {"lors": int(out[0]), "lists_differ": int(out[1]), "max_rel_length": float(out[2]),
                "max_rel_line": float(out[3]), "rms_rel_line": float(out[4])}

    def bin_coordinates(self, p: ProjSpec, pairs):
        """[n, 5]: flag, seg, view, axial, tang of each (ring1, crystal1,
        ring2, crystal2) pair (zeros where the flag is 0)."""
        f = self.proj(p)
        pairs = np.asarray(pairs, np.int64).reshape(-1, 4)
        out = np.zeros((pairs.shape[0], 5), np.int32)
        o = [C.c_int() for _ in range(4)]
        for i, (r1, c1, r2, c2) in enumerate(pairs):
            if self.L.fo_bin_coordinates(C.byref(f), int(r1), int(c1), int(r2), int(c2), *[C.byref(x) for x in o]):
                out[i] = (1, o[0].value, o[1].value, o[2].value, o[3].value)
        return out

    def rebin_weight(self, p: ProjSpec, sino):
        out = np.ascontiguousarray(sino, np.float32).copy()
        self.L.fo_rebin_weight(C.byref(self.proj(p)), out)
        return out

    def em_update(self, img, bp, sens):
        img = np.ascontiguousarray(img, np.float32).copy()
        bp = np.ascontiguousarray(bp, np.float32).copy()
        self.L.fo_em_update(img.size, img.ravel(), bp.ravel(), np.ascontiguousarray(sens, np.float32).ravel())
        return img, bp

    def convolve(self, v: VolSpec, img, fwhm, cut_radius=0.0):
        out = np.ascontiguousarray(img, np.float32).copy()
        self.L.fo_convolve(C.byref(fo_vol(v)), out.ravel(), np.asarray(fwhm, np.float32), float(cut_radius))
        return out

    def cut_circle(self, v: VolSpec, img, cut_radius):
        out = np.ascontiguousarray(img, np.float32).copy()
        self.L.fo_cut_circle(C.byref(fo_vol(v)), out.ravel(), float(cut_radius))
        return out

    def apply_mask(self, img, mask):
        out = np.ascontiguousarray(img, np.float32).copy()
        self.L.fo_apply_mask(out.size, out.ravel(), np.ascontiguousarray(mask, np.float32).ravel())
        return out

    def hu_to_mu(self, img):
        out = np.ascontiguousarray(img, np.float32).copy()
        self.L.fo_hu_to_mu(out.size, out.ravel())
        return out

    def exponential(self, sino):
        out = np.ascontiguousarray(sino, np.float32).copy()
        self.L.fo_exponential(out.size, out)
        return out

    def proj_multiply(self, a, b):
        out = np.ascontiguousarray(a, np.float32).copy()
        self.L.fo_proj_multiply(out.size, out, np.ascontiguousarray(b, np.float32))
        return out


# --------------------------------------------------------------- reference

class RefVol(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("vx", C.c_double), ("vy", C.c_double), ("vz", C.c_double),
        ("ox", C.c_double), ("oy", C.c_double), ("oz", C.c_double),
        ("nframes", C.c_int),
    ]


def ref_vol(v: VolSpec) -> RefVol:
    return RefVol(int(v.size[0]), int(v.size[1]), int(v.size[2]),
                  float(v.voxel[0]), float(v.voxel[1]), float(v.voxel[2]),
                  float(v.offset[0]), float(v.offset[1]), float(v.offset[2]), int(v.n_frames))


class Reference:
    """FIR's own compiled code, driven through its C++ API by ref_harness.cc."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle reference)")
        L = C.CDLL(path)
        self.L = L
        L.ref_last_error.restype = C.c_char_p
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_siddon_paths.argtypes = [C.POINTER(RefVol), C.c_int, _f64p, C.c_int, _i32p, _f64p, _i32p, _i32p]
        L.ref_scanner_tables.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, _f64p, _f64p, C.c_int, C.c_int]
        L.ref_proj_geometry.argtypes = [C.c_char_p, _i32p, C.c_int]
        L.ref_lor_table.argtypes = [C.c_char_p, _i32p]
        L.ref_path_counts.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(RefVol), _i32p]
        L.ref_forward.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(RefVol), _f32p, _f32p]
        L.ref_backward.argtypes = [C.c_char_p, C.c_char_p, _f32p, C.POINTER(RefVol), C.c_int, _f32p]
        L.ref_sensitivity.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(RefVol), C.c_int, _f32p]
        L.ref_osem.argtypes = [C.c_char_p, C.c_char_p, _f32p, C.c_void_p, C.POINTER(RefVol), _f32p, _f32p,
                               C.c_int, C.c_int, C.c_float, C.c_int, _f32p, C.c_int, C.c_char_p]
        L.ref_osem_reso_reco.argtypes = [C.c_char_p, C.c_char_p, _f32p, C.c_void_p, C.POINTER(RefVol), _f32p,
                                         _f32p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _f32p, C.c_char_p]
        L.ref_convolve.argtypes = [C.POINTER(RefVol), _f32p, _f32p, C.c_float]
        L.ref_cut_circle.argtypes = [C.POINTER(RefVol), _f32p, C.c_float]
        L.ref_apply_mask.argtypes = [C.POINTER(RefVol), _f32p, _f32p]
        L.ref_hu_to_mu.argtypes = [C.POINTER(RefVol), _f32p]
        L.ref_proj_exponential.argtypes = [C.c_char_p, _f32p]
        L.ref_proj_multiply.argtypes = [C.c_char_p, _f32p, _f32p]
        L.ref_bin_coordinates.argtypes = [C.c_char_p, C.c_longlong, C.c_void_p, C.c_void_p]
        L.ref_rebin_weight.argtypes = [C.c_char_p, _f32p]
        L.ref_em_update.argtypes = [C.POINTER(RefVol), _f32p, _f32p, _f32p]
        self.tmp = tempfile.mkdtemp(prefix="firref_")
        self._n = 0

    def threads(self, n: int) -> None:
        self.L.ref_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.L.ref_get_threads())

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.ref_last_error().decode())

    def _files(self, s: Optional[ScannerSpec], p: Optional[ProjSpec]):
        self._n += 1
        sp = hp = None
        if s is not None:
            sp = os.path.join(self.tmp, f"s{self._n}.scan")
            interfile.write_scanner(sp, s)
        if p is not None:
            hp = os.path.join(self.tmp, f"p{self._n}.hs")
            interfile.write_proj_header(hp, p)
        return (sp.encode() if sp else None), (hp.encode() if hp else None)

    def siddon_paths(self, v: VolSpec, pts: np.ndarray):
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 6)
        n = pts.shape[0]
        cap = int(v.size[0] + v.size[1] + v.size[2] + 2)
        coords = np.full((n, cap), -1, np.int32)
        lengths = np.zeros((n, cap), np.float64)
        counts = np.zeros(n, np.int32)
        crosses = np.zeros(n, np.int32)
        self._check(self.L.ref_siddon_paths(C.byref(ref_vol(v)), n, pts.ravel(), cap, coords.ravel(),
                                            lengths.ravel(), counts, crosses))
        return crosses, counts, coords, lengths

    def scanner_tables(self, s: ScannerSpec):
        sp, _ = self._files(s, None)
        xy = np.zeros(2 * s.n_crystals_per_ring, np.float64)
        z = np.zeros(2 * s.n_rings - 1, np.float64)
        self._check(self.L.ref_scanner_tables(sp, None, None, xy, z, s.n_crystals_per_ring, 2 * s.n_rings - 1))
        return xy, z

    def proj_geometry(self, p: ProjSpec):
        _, hp = self._files(None, p)
        out = np.zeros(7 + p.n_segments, np.int32)
        self._check(self.L.ref_proj_geometry(hp, out, out.size))
        keys = ["n_bins", "seg_offset", "tang_offset", "n_views", "half_span", "max_ring_diff", "n_tang_coords"]
        d = {k: int(out[i]) for i, k in enumerate(keys)}
        d["n_axial"] = [int(x) for x in out[7:]]
        return d

    def lor_table(self, p: ProjSpec, n_bins: int):
        _, hp = self._files(None, p)
        out = np.zeros((n_bins, 4), np.int32)
        self._check(self.L.ref_lor_table(hp, out.ravel()))
        return out

    def path_counts(self, s, p, v: VolSpec, n_bins: int):
        """Elements of FIR's Siddon path for every bin (file order), all threads."""
        sp, hp = self._files(s, p)
        out = np.zeros(n_bins, np.int32)
        self._check(self.L.ref_path_counts(sp, hp, C.byref(ref_vol(v)), out))
        return out

    def forward(self, s, p, v: VolSpec, img, n_bins: int):
        sp, hp = self._files(s, p)
        out = np.zeros(n_bins, np.float32)
        self._check(self.L.ref_forward(sp, hp, C.byref(ref_vol(v)), np.ascontiguousarray(img, np.float32).ravel(),
                                       out))
        return out

    def backward(self, s, p, v: VolSpec, sino, n_subsets: int = 1):
        sp, hp = self._files(s, p)
        out = np.zeros(v.n_voxels * n_subsets, np.float32)
        self._check(self.L.ref_backward(sp, hp, np.ascontiguousarray(sino, np.float32), C.byref(ref_vol(v)),
                                        n_subsets, out))
        return out.reshape(n_subsets * v.size[2], v.size[1], v.size[0])

    def sensitivity(self, s, p, v: VolSpec, n_subsets: int = 1):
        sp, hp = self._files(s, p)
        out = np.zeros(v.n_voxels * n_subsets, np.float32)
        self._check(self.L.ref_sensitivity(sp, hp, C.byref(ref_vol(v)), n_subsets, out))
        return out.reshape(n_subsets * v.size[2], v.size[1], v.size[0])

    def osem(self, s, p, v: VolSpec, sino, img, sens, prm: OSEMParams, bias=None):
        sp, hp = self._files(s, p)
        img = np.ascontiguousarray(img, np.float32).copy().ravel()
        bias_arr = None if bias is None else np.ascontiguousarray(bias, np.float32)
        bptr = None if bias_arr is None else bias_arr.ctypes.data_as(C.c_void_p)
        out_name = os.path.join(self.tmp, f"osem{self._n}").encode()
        self._check(self.L.ref_osem(sp, hp, np.ascontiguousarray(sino, np.float32), bptr, C.byref(ref_vol(v)), img,
                                    np.ascontiguousarray(sens, np.float32).ravel(), prm.n_iterations,
                                    prm.n_subsets, prm.cut_radius, prm.convolution_interval,
                                    np.asarray(prm.fwhm_xyz, np.float32), prm.save_interval, out_name))
        return img.reshape(v.shape_zyx)

    def osem_reso_reco(self, s, p, v: VolSpec, sino, img, sens, prm: OSEMParams, bias=None):
        """FIR's reconAlgos::OSEM_ResoReco; returns (image, sens), FIR having
        filtered every frame of the sensitivity in place."""
        sp, hp = self._files(s, p)
        img = np.ascontiguousarray(img, np.float32).copy().ravel()
        sens = np.ascontiguousarray(sens, np.float32).copy().ravel()
        bias_arr = None if bias is None else np.ascontiguousarray(bias, np.float32)
        bptr = None if bias_arr is None else bias_arr.ctypes.data_as(C.c_void_p)
        out_name = os.path.join(self.tmp, f"reso{self._n}").encode()
        self._check(self.L.ref_osem_reso_reco(sp, hp, np.ascontiguousarray(sino, np.float32), bptr,
                                              C.byref(ref_vol(v)), img, sens, sens.size // v.n_voxels,
                                              prm.n_iterations, prm.n_subsets, prm.cut_radius,
                                              prm.convolution_interval, np.asarray(prm.fwhm_xyz, np.float32),
                                              out_name))
        return img.reshape(v.shape_zyx), sens

    def convolve(self, v: VolSpec, img, fwhm, cut_radius=0.0):
        out = np.ascontiguousarray(img, np.float32).copy()
        self._check(self.L.ref_convolve(C.byref(ref_vol(v)), out.ravel(), np.asarray(fwhm, np.float32),
                                        float(cut_radius)))
        return out

    def cut_circle(self, v: VolSpec, img, cut_radius):
        out = np.ascontiguousarray(img, np.float32).copy()
        self._check(self.L.ref_cut_circle(C.byref(ref_vol(v)), out.ravel(), float(cut_radius)))
        return out

    def apply_mask(self, v: VolSpec, img, mask):
        out = np.ascontiguousarray(img, np.float32).copy()
        self._check(self.L.ref_apply_mask(C.byref(ref_vol(v)), out.ravel(),
                                          np.ascontiguousarray(mask, np.float32).ravel()))
        return out

    def hu_to_mu(self, v: VolSpec, img):
        out = np.ascontiguousarray(img, np.float32).copy()
        self._check(self.L.ref_hu_to_mu(C.byref(ref_vol(v)), out.ravel()))
        return out

    def exponential(self, p: ProjSpec, sino):
        _, hp = self._files(None, p)
        out = np.ascontiguousarray(sino, np.float32).copy()
        self._check(self.L.ref_proj_exponential(hp, out))
        return out

    def proj_multiply(self, p: ProjSpec, a, b):
        _, hp = self._files(None, p)
        out = np.ascontiguousarray(a, np.float32).copy()
        self._check(self.L.ref_proj_multiply(hp, out, np.ascontiguousarray(b, np.float32)))
        return out

    def bin_coordinates(self, p: ProjSpec, pairs):
        _, hp = self._files(None, p)
        pairs = np.ascontiguousarray(np.asarray(pairs, np.int32).reshape(-1, 4))
        out = np.zeros((pairs.shape[0], 5), np.int32)
        self._check(self.L.ref_bin_coordinates(hp, pairs.shape[0], pairs.ctypes.data, out.ctypes.data))
        return out

    def rebin_weight(self, p: ProjSpec, sino):
        _, hp = self._files(None, p)
        out = np.ascontiguousarray(sino, np.float32).copy()
        self._check(self.L.ref_rebin_weight(hp, out))
        return out

    def em_update(self, v: VolSpec, img, bp, sens):
        img = np.ascontiguousarray(img, np.float32).copy()
        bp = np.ascontiguousarray(bp, np.float32).copy()
        self._check(self.L.ref_em_update(C.byref(ref_vol(v)), img.ravel(), bp.ravel(),
                                         np.ascontiguousarray(sens, np.float32).ravel()))
        return img, bp
