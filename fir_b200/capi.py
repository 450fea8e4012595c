"""ctypes binding of the C ABI in ``include/fir_cuda.h``.

Loads ``fir_b200/lib/libfir_cuda.so`` (built in-tree by ``fir_b200.build``).
There is no fallback: if the library is missing or no GPU is present, calls
raise.  Data arguments may be CUDA torch tensors (device pointers, work is
enqueued on torch's current stream) or numpy arrays / CPU tensors (host
pointers, the library stages them and the call is synchronous).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from .geometry import OSEMParams, ProjSpec, ScannerSpec, VolSpec

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libfir_cuda.so")

FIR_OK = 0
FIR_OPT_GEOMETRY = 1
FIR_OPT_BACKPROJ_MODE = 2
FIR_OPT_SKIP_ZERO_BINS = 3
FIR_OPT_BLOCK_SIZE = 4
FIR_OPT_TIMING = 5
FIR_OPT_DETERMINISTIC_CHUNK = 6
FIR_OPT_STEP_LIMIT = 7
FIR_OPT_TRAVERSAL = 8
FIR_TRAVERSAL_EXACT = 0
FIR_TRAVERSAL_FLOAT = 1
FIR_GEOMETRY_REFERENCE = 0
FIR_GEOMETRY_EXACT = 1
FIR_BACKPROJ_ATOMIC = 0
FIR_BACKPROJ_DETERMINISTIC = 1
FIR_F32 = 0
FIR_F64 = 1


class FirError(RuntimeError):
    """A C-ABI call returned a non-zero fir_status."""

    def __init__(self, status: int, name: str, message: str):
        super().__init__(f"{name}: {message}")
        self.status = status
        self.name = name


class VolDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("voxel_x", C.c_double), ("voxel_y", C.c_double), ("voxel_z", C.c_double),
        ("offset_x", C.c_double), ("offset_y", C.c_double), ("offset_z", C.c_double),
        ("n_frames", C.c_int),
    ]


class ProjDesc(C.Structure):
    _fields_ = [
        ("n_rings", C.c_int), ("n_crystals_per_ring", C.c_int), ("segment_span", C.c_int),
        ("n_segments", C.c_int), ("n_tang_coords", C.c_int),
    ]


class ProjInfo(C.Structure):
    _fields_ = [
        ("n_bins", C.c_longlong), ("seg_offset", C.c_int), ("tang_offset", C.c_int),
        ("n_views", C.c_int), ("half_span", C.c_int), ("max_ring_diff", C.c_int),
        ("n_tang_coords", C.c_int),
    ]


class ScannerDesc(C.Structure):
    _fields_ = [
        ("crystal_dims", C.c_double * 3), ("crystal_repeat", C.c_int * 2),
        ("inter_crystal", C.c_double * 2), ("module_dims", C.c_double * 3),
        ("module_repeat", C.c_int * 2), ("inter_module", C.c_double * 2),
        ("rsector_dims", C.c_double * 3), ("rsector_repeat", C.c_int),
        ("rsector_inner_radius", C.c_double),
    ]


class OsemParamsDesc(C.Structure):
    _fields_ = [
        ("n_iterations", C.c_int), ("n_subsets", C.c_int), ("save_interval", C.c_int),
        ("cut_radius", C.c_float), ("convolution_interval", C.c_int), ("fwhm_xyz", C.c_float * 3),
    ]


SAVE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.POINTER(C.c_float))

_lib = None

_SIGS = {
    "fir_abi_version": (C.c_int, []),
    "fir_last_error": (C.c_char_p, []),
    "fir_status_string": (C.c_char_p, [C.c_int]),
    "fir_proj_geometry": (C.c_int, [C.POINTER(ProjDesc), C.POINTER(ProjInfo), C.c_void_p]),
    "fir_scanner_tables": (C.c_int, [C.POINTER(ScannerDesc), C.c_void_p, C.c_void_p, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    "fir_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "fir_ctx_destroy": (C.c_int, [C.c_void_p]),
    "fir_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fir_ctx_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "fir_ctx_get_option": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "fir_ctx_set_scanner": (C.c_int, [C.c_void_p, C.POINTER(ScannerDesc)]),
    "fir_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "fir_ctx_launch_count": (C.c_longlong, [C.c_void_p]),
    "fir_ctx_projector_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_int]),
    "fir_forward": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.POINTER(ProjDesc), C.c_void_p]),
    "fir_forward_exp": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.POINTER(ProjDesc), C.c_void_p]),
    "fir_backward": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.POINTER(VolDesc), C.c_void_p,
                               C.c_int]),
    "fir_sensitivity": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.POINTER(VolDesc), C.c_void_p, C.c_int]),
    "fir_osem_subiteration": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p,
                                        C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.POINTER(OsemParamsDesc),
                                        C.c_int, C.c_int]),
    "fir_osem": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p, C.POINTER(VolDesc),
                           C.c_void_p, C.c_void_p, C.POINTER(OsemParamsDesc), C.c_void_p, C.c_void_p]),
    "fir_osem_psf": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p, C.POINTER(VolDesc),
                               C.c_void_p, C.c_void_p, C.POINTER(OsemParamsDesc), C.c_void_p, C.c_void_p]),
    "fir_osem_reso_reco": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p,
                                     C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.c_int,
                                     C.POINTER(OsemParamsDesc), C.c_void_p, C.c_void_p]),
    "fir_osem_weighted": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.POINTER(OsemParamsDesc),
                                    C.c_void_p, C.c_void_p]),
    "fir_osem_subiteration_noalloc": (C.c_int, [C.POINTER(ProjDesc), C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.c_void_p,
                                                C.POINTER(OsemParamsDesc), C.c_int, C.c_int, C.c_int,
                                                C.c_void_p]),
    "fir_ratio_backprojection": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p,
                                           C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "fir_ratio_backprojection_shard": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p,
                                                 C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                 C.c_int, C.c_int]),
    "fir_em_update": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.c_void_p, C.c_void_p]),
    "fir_convolve": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.POINTER(C.c_float), C.c_float]),
    "fir_cut_circle": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.c_float]),
    "fir_apply_mask": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.c_void_p]),
    "fir_hu_to_mu": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p]),
    "fir_proj_exponential": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p]),
    "fir_proj_multiply": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.c_void_p]),
    "fir_siddon_paths": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_longlong, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fir_lor_paths": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.POINTER(VolDesc), C.c_longlong, C.c_void_p,
                                C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fir_forward_frames": (C.c_int, [C.c_void_p, C.POINTER(VolDesc), C.c_void_p, C.POINTER(ProjDesc), C.c_void_p,
                                     C.c_int]),
    "fir_backward_frames": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p, C.POINTER(VolDesc), C.c_void_p,
                                      C.c_int]),
    "fir_bin_coordinates": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_longlong, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "fir_proj_rebin_weight": (C.c_int, [C.c_void_p, C.POINTER(ProjDesc), C.c_void_p]),
    "fir_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.POINTER(ScannerDesc),
                                   C.POINTER(ProjDesc), C.POINTER(VolDesc), C.POINTER(OsemParamsDesc)]),
    "fir_batch_destroy": (C.c_int, [C.c_void_p]),
    "fir_batch_set_data": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fir_batch_set_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "fir_batch_get_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "fir_batch_set_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "fir_batch_get_launch": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fir_batch_tune": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "fir_batch_tune_report": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.POINTER(C.c_int)]),
    "fir_batch_set_bundle": (C.c_int, [C.c_void_p, C.c_int]),
    "fir_batch_get_bundle": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "fir_batch_schedule": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "fir_batch_osem": (C.c_int, [C.c_void_p, C.c_int]),
}


def exported_symbols():
    """Names of every entry point this binding declares (all of fir_cuda.h)."""
    return sorted(_SIGS)


def lib():
    """The loaded C-ABI library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m fir_b200.build` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != FIR_OK:
        L = lib()
        raise FirError(status, L.fir_status_string(status).decode(), L.fir_last_error().decode())


# ----------------------------------------------------------- descriptors

def vol_desc(v: VolSpec, n_frames: Optional[int] = None) -> VolDesc:
    return VolDesc(int(v.size[0]), int(v.size[1]), int(v.size[2]),
                   float(v.voxel[0]), float(v.voxel[1]), float(v.voxel[2]),
                   float(v.offset[0]), float(v.offset[1]), float(v.offset[2]),
                   int(v.n_frames if n_frames is None else n_frames))


def proj_desc(p: ProjSpec) -> ProjDesc:
    return ProjDesc(int(p.n_rings), int(p.n_crystals_per_ring), int(p.segment_span), int(p.n_segments),
                    int(p.n_tang_coords))


def scanner_desc(s: ScannerSpec) -> ScannerDesc:
    d = ScannerDesc()
    d.crystal_dims[:] = [float(x) for x in s.crystal_dims]
    d.crystal_repeat[:] = [int(x) for x in s.crystal_repeat]
    d.inter_crystal[:] = [float(x) for x in s.inter_crystal]
    d.module_dims[:] = [float(x) for x in s.module_dims]
    d.module_repeat[:] = [int(x) for x in s.module_repeat]
    d.inter_module[:] = [float(x) for x in s.inter_module]
    d.rsector_dims[:] = [float(x) for x in s.rsector_dims]
    d.rsector_repeat = int(s.rsector_repeat_number)
    d.rsector_inner_radius = float(s.rsector_inner_radius)
    return d


def osem_desc(p: OSEMParams) -> OsemParamsDesc:
    d = OsemParamsDesc(int(p.n_iterations), int(p.n_subsets), int(p.save_interval), float(p.cut_radius),
                       int(p.convolution_interval))
    d.fwhm_xyz[:] = [float(x) for x in p.fwhm_xyz]
    return d


def proj_geometry(p: ProjSpec) -> dict:
    """``ProjHeader::check`` + ``ProjGeometry::fill`` as a dict."""
    info = ProjInfo()
    n_axial = (C.c_int * max(1, int(p.n_segments)))()
    _check(lib().fir_proj_geometry(C.byref(proj_desc(p)), C.byref(info), C.cast(n_axial, C.c_void_p)))
    return {
        "n_bins": int(info.n_bins), "seg_offset": info.seg_offset, "tang_offset": info.tang_offset,
        "n_views": info.n_views, "half_span": info.half_span, "max_ring_diff": info.max_ring_diff,
        "n_tang_coords": info.n_tang_coords, "n_axial": [int(x) for x in n_axial][: int(p.n_segments)],
    }


def scanner_tables(s: ScannerSpec):
    """Crystal XY (``[n_crystals_per_ring, 2]``) and slice Z (``[2*n_rings-1]``) tables."""
    nr, nc = C.c_int(), C.c_int()
    d = scanner_desc(s)
    _check(lib().fir_scanner_tables(C.byref(d), None, None, C.byref(nr), C.byref(nc)))
    xy = np.zeros((nc.value, 2), np.float64)
    z = np.zeros(2 * nr.value - 1, np.float64)
    _check(lib().fir_scanner_tables(C.byref(d), xy.ctypes.data, z.ctypes.data, None, None))
    return xy, z


# ------------------------------------------------------------- buffers

def _ptr(x, dtype=np.float32, writable=False, n: Optional[int] = None):
    """Data pointer of a torch tensor or numpy array, after dtype/layout checks."""
    if x is None:
        return None
    try:
        import torch

        if isinstance(x, torch.Tensor):
            tdt = {np.float32: torch.float32, np.float64: torch.float64, np.int32: torch.int32,
                   np.int64: torch.int64}[dtype]
            if x.dtype != tdt or not x.is_contiguous():
                raise TypeError(f"expected a contiguous {tdt} tensor, got {x.dtype} "
                                f"(contiguous={x.is_contiguous()})")
            if n is not None and x.numel() < n:
                raise ValueError(f"buffer holds {x.numel()} elements, {n} required")
            return x.data_ptr()
    except ImportError:
        pass
    if not isinstance(x, np.ndarray):
        raise TypeError(f"expected a numpy array or torch tensor, got {type(x)}")
    if x.dtype != np.dtype(dtype) or not x.flags["C_CONTIGUOUS"]:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype)} array, got {x.dtype}")
    if writable and not x.flags["WRITEABLE"]:
        raise ValueError("output array is read-only")
    if n is not None and x.size < n:
        raise ValueError(f"buffer holds {x.size} elements, {n} required")
    return x.ctypes.data


def _dtype_of(x):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return np.float64 if x.dtype == torch.float64 else np.float32
    except ImportError:
        pass
    return np.float64 if np.asarray(x).dtype == np.float64 else np.float32


class Context:
    """A ``fir_ctx``: one device, one stream, scanner tables and scratch."""

    def __init__(self, scanner: Optional[ScannerSpec] = None, device: int = 0):
        self._h = C.c_void_p()
        _check(lib().fir_ctx_create(C.byref(self._h), int(device)))
        self.device = int(device)
        self.scanner = None
        if scanner is not None:
            self.set_scanner(scanner)

    def close(self) -> None:
        if self._h:
            lib().fir_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- configuration
    def set_scanner(self, s: ScannerSpec) -> None:
        _check(lib().fir_ctx_set_scanner(self._h, C.byref(scanner_desc(s))))
        self.scanner = s

    def set_option(self, opt: int, value: int) -> None:
        _check(lib().fir_ctx_set_option(self._h, int(opt), int(value)))

    def get_option(self, opt: int) -> int:
        v = C.c_int()
        _check(lib().fir_ctx_get_option(self._h, int(opt), C.byref(v)))
        return v.value

    def set_stream(self, stream_handle: int) -> None:
        _check(lib().fir_ctx_set_stream(self._h, C.c_void_p(int(stream_handle))))

    def use_torch_stream(self) -> None:
        import torch

        self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def synchronize(self) -> None:
        _check(lib().fir_ctx_synchronize(self._h))

    @property
    def launch_count(self) -> int:
        return int(lib().fir_ctx_launch_count(self._h))

    def projector_time(self, reset: bool = True):
        """(device ms, launches) of projector kernels since the last reset
        (needs ``set_option(FIR_OPT_TIMING, 1)``)."""
        ms, n = C.c_double(), C.c_longlong()
        _check(lib().fir_ctx_projector_time(self._h, C.byref(ms), C.byref(n), int(reset)))
        return ms.value, n.value

    def _prep(self, *bufs):
        # keep torch's stream semantics when device tensors are involved
        try:
            import torch

            if any(isinstance(b, torch.Tensor) and b.is_cuda for b in bufs if b is not None):
                self.use_torch_stream()
        except ImportError:
            pass

    # -- projectors
    def forward(self, vol: VolSpec, img, proj: ProjSpec, sino) -> None:
        self._prep(img, sino)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_forward(self._h, C.byref(vol_desc(vol, 1)), _ptr(img, n=vol.n_voxels),
                                 C.byref(proj_desc(proj)), _ptr(sino, writable=True, n=nb)))

    def forward_exp(self, vol: VolSpec, mu, proj: ProjSpec, acf) -> None:
        self._prep(mu, acf)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_forward_exp(self._h, C.byref(vol_desc(vol, 1)), _ptr(mu, n=vol.n_voxels),
                                     C.byref(proj_desc(proj)), _ptr(acf, writable=True, n=nb)))

    def backward(self, proj: ProjSpec, sino, vol: VolSpec, img, n_subsets: int = 1) -> None:
        self._prep(sino, img)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_backward(self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb),
                                  C.byref(vol_desc(vol, n_subsets)),
                                  _ptr(img, writable=True, n=vol.n_voxels * n_subsets), int(n_subsets)))

    def sensitivity(self, proj: ProjSpec, vol: VolSpec, sens, n_subsets: int = 1) -> None:
        self._prep(sens)
        _check(lib().fir_sensitivity(self._h, C.byref(proj_desc(proj)), C.byref(vol_desc(vol, n_subsets)),
                                     _ptr(sens, writable=True, n=vol.n_voxels * n_subsets), int(n_subsets)))

    def osem_subiteration(self, proj: ProjSpec, sino, vol: VolSpec, img, sens_frame, params: OSEMParams,
                          subset: int, subiter: int, bias=None) -> None:
        self._prep(sino, img, sens_frame, bias)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_osem_subiteration(self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb),
                                           _ptr(bias, n=nb), C.byref(vol_desc(vol, 1)),
                                           _ptr(img, writable=True, n=vol.n_voxels),
                                           _ptr(sens_frame, n=vol.n_voxels), C.byref(osem_desc(params)),
                                           int(subset), int(subiter)))

    def osem(self, proj: ProjSpec, sino, vol: VolSpec, img, sens, params: OSEMParams, bias=None,
             save=None, psf: bool = False, mult=None) -> None:
        """reconAlgos::OSEM (``psf``: the resolution-modelling form,
        ``fir_osem_psf``; ``mult``: per-bin multiplicative factors of the
        ordinary-Poisson model, ``fir_osem_weighted``, with sens = A_s^T mult).
        ``save(subiter, image_numpy)`` is called at the save interval."""
        self._prep(sino, img, sens, bias, mult)
        nb = proj_geometry(proj)["n_bins"]
        cb = None
        if save is not None:
            shape = vol.shape_zyx

            def _cb(user, subiter, ptr):
                arr = np.ctypeslib.as_array(ptr, shape=(vol.n_voxels,)).copy().reshape(shape)
                save(int(subiter), arr)

            cb = SAVE_FN(_cb)
        if mult is not None:
            if psf:
                raise ValueError("psf and mult cannot be combined")
            _check(lib().fir_osem_weighted(self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb), _ptr(mult, n=nb),
                                           _ptr(bias, n=nb), C.byref(vol_desc(vol, 1)),
                                           _ptr(img, writable=True, n=vol.n_voxels),
                                           _ptr(sens, n=vol.n_voxels * params.n_subsets), C.byref(osem_desc(params)),
                                           C.cast(cb, C.c_void_p) if cb is not None else None, None))
            return
        fn = lib().fir_osem_psf if psf else lib().fir_osem
        _check(fn(self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb), _ptr(bias, n=nb),
                  C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=vol.n_voxels),
                  _ptr(sens, n=vol.n_voxels * params.n_subsets), C.byref(osem_desc(params)),
                  C.cast(cb, C.c_void_p) if cb is not None else None, None))

    def osem_reso_reco(self, proj: ProjSpec, sino, vol: VolSpec, img, sens, params: OSEMParams,
                       n_sens_frames: Optional[int] = None, bias=None) -> None:
        """reconAlgos::OSEM_ResoReco as FIR runs it (``fir_osem_reso_reco``):
        every frame of ``sens`` (``n_sens_frames``, default the number of
        subsets) is filtered in place once, then every sub-iteration divides
        the image by the subset's sensitivity frame and multiplies it by the
        filtered backprojection of the unfiltered image's ratio."""
        self._prep(sino, img, sens, bias)
        nb = proj_geometry(proj)["n_bins"]
        nf = int(params.n_subsets if n_sens_frames is None else n_sens_frames)
        _check(lib().fir_osem_reso_reco(self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb), _ptr(bias, n=nb),
                                        C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=vol.n_voxels),
                                        _ptr(sens, writable=True, n=vol.n_voxels * nf), nf,
                                        C.byref(osem_desc(params)), None, None))

    def ratio_backprojection(self, proj: ProjSpec, sino, vol: VolSpec, img, bp, n_subsets: int = 1,
                             subset: int = 0, bias=None, n_shards: int = 1, shard: int = 0) -> None:
        """bp <- backprojection of sino / (projection of img + bias) over one
        subset, or over shard ``shard`` of ``n_shards`` of its views (the
        subset's k-th view with k % n_shards == shard)."""
        self._prep(sino, img, bp, bias)
        nb = proj_geometry(proj)["n_bins"]
        args = (self._h, C.byref(proj_desc(proj)), _ptr(sino, n=nb), _ptr(bias, n=nb), C.byref(vol_desc(vol, 1)),
                _ptr(img, n=vol.n_voxels), _ptr(bp, writable=True, n=vol.n_voxels), int(n_subsets), int(subset))
        if n_shards == 1:
            _check(lib().fir_ratio_backprojection(*args))
        else:
            _check(lib().fir_ratio_backprojection_shard(*args, int(n_shards), int(shard)))

    # -- image / sinogram operations
    def em_update(self, vol: VolSpec, img, bp, sens_frame) -> None:
        self._prep(img, bp, sens_frame)
        n = vol.n_voxels
        _check(lib().fir_em_update(self._h, C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=n),
                                   _ptr(bp, writable=True, n=n), _ptr(sens_frame, n=n)))

    def convolve(self, vol: VolSpec, img, fwhm: Sequence[float], cut_radius: float = 0.0) -> None:
        self._prep(img)
        f = (C.c_float * 3)(*[float(x) for x in fwhm])
        _check(lib().fir_convolve(self._h, C.byref(vol_desc(vol)), _ptr(img, writable=True,
                                                                        n=vol.n_voxels * vol.n_frames),
                                  f, float(cut_radius)))

    def cut_circle(self, vol: VolSpec, img, cut_radius: float) -> None:
        self._prep(img)
        _check(lib().fir_cut_circle(self._h, C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=vol.n_voxels),
                                    float(cut_radius)))

    def apply_mask(self, vol: VolSpec, img, mask) -> None:
        self._prep(img, mask)
        _check(lib().fir_apply_mask(self._h, C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=vol.n_voxels),
                                    _ptr(mask, n=vol.n_voxels)))

    def hu_to_mu(self, vol: VolSpec, img) -> None:
        self._prep(img)
        _check(lib().fir_hu_to_mu(self._h, C.byref(vol_desc(vol, 1)), _ptr(img, writable=True, n=vol.n_voxels)))

    def proj_exponential(self, proj: ProjSpec, sino) -> None:
        self._prep(sino)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_proj_exponential(self._h, C.byref(proj_desc(proj)), _ptr(sino, writable=True, n=nb)))

    def proj_multiply(self, proj: ProjSpec, a, b) -> None:
        self._prep(a, b)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_proj_multiply(self._h, C.byref(proj_desc(proj)), _ptr(a, writable=True, n=nb),
                                       _ptr(b, n=nb)))

    # -- path dumps
    def _frames_args(self, vol: VolSpec, img, proj: ProjSpec, sino):
        n_frames = img.shape[0] if img.ndim == 4 else 1
        dt = np.float64 if _dtype_of(img) == np.float64 else np.float32
        if _dtype_of(sino) != dt:
            raise TypeError("image and sinogram must have the same dtype")
        nb = proj_geometry(proj)["n_bins"]
        return (vol_desc(vol, n_frames), _ptr(img, dt, n=vol.n_voxels * n_frames), _ptr(sino, dt, n=nb * n_frames),
                FIR_F64 if dt == np.float64 else FIR_F32)

    def forward_frames(self, vol: VolSpec, img, proj: ProjSpec, sino) -> None:
        """sino[f] = projection of img[f] for every frame ([F, nz, ny, nx] ->
        [F, n_bins]); float32 (FIR's arithmetic) or float64."""
        self._prep(img, sino)
        vd, pi, ps, dt = self._frames_args(vol, img, proj, sino)
        _check(lib().fir_forward_frames(self._h, C.byref(vd), pi, C.byref(proj_desc(proj)), ps, dt))

    def backward_frames(self, proj: ProjSpec, sino, vol: VolSpec, img) -> None:
        """img[f] = backprojection of sino[f] (the adjoint of forward_frames)."""
        self._prep(img, sino)
        vd, pi, ps, dt = self._frames_args(vol, img, proj, sino)
        _check(lib().fir_backward_frames(self._h, C.byref(proj_desc(proj)), ps, C.byref(vd), pi, dt))

    def bin_coordinates(self, proj: ProjSpec, pairs):
        """ProjData::getBinCoordinates of n (ring1, crystal1, ring2, crystal2)
        pairs: returns (coords [n, 5] = found, seg, view, axial, tang; bins [n]
        flat index or -1)."""
        pairs = np.ascontiguousarray(np.asarray(pairs, np.int32).reshape(-1, 4))
        n = pairs.shape[0]
        coords = np.zeros((n, 5), np.int32)
        bins = np.zeros(n, np.int64)
        _check(lib().fir_bin_coordinates(self._h, C.byref(proj_desc(proj)), n, pairs.ctypes.data,
                                         coords.ctypes.data, bins.ctypes.data))
        return coords, bins

    def proj_rebin_weight(self, proj: ProjSpec, sino) -> None:
        """ProjData::rebinWeight in place."""
        self._prep(sino)
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_proj_rebin_weight(self._h, C.byref(proj_desc(proj)), _ptr(sino, writable=True, n=nb)))

    def siddon_paths(self, vol: VolSpec, ends, cap: Optional[int] = None):
        ends = np.ascontiguousarray(ends, np.float64).reshape(-1, 6)
        n = ends.shape[0]
        cap = int(cap if cap is not None else vol.size[0] + vol.size[1] + vol.size[2] + 2)
        coords = np.full((n, cap), -1, np.int32)
        lengths = np.zeros((n, cap), np.float64)
        counts = np.zeros(n, np.int32)
        crosses = np.zeros(n, np.int32)
        _check(lib().fir_siddon_paths(self._h, C.byref(vol_desc(vol, 1)), n, ends.ctypes.data, cap,
                                      coords.ctypes.data, lengths.ctypes.data, counts.ctypes.data,
                                      crosses.ctypes.data))
        return crosses, counts, coords, lengths

    def lor_paths(self, proj: ProjSpec, vol: VolSpec, bins, cap: Optional[int] = None):
        bins = np.ascontiguousarray(bins, np.int64).ravel()
        n = bins.size
        cap = int(cap if cap is not None else vol.size[0] + vol.size[1] + vol.size[2] + 2)
        coords = np.full((n, cap), -1, np.int32)
        lengths = np.zeros((n, cap), np.float64)
        counts = np.zeros(n, np.int32)
        crosses = np.zeros(n, np.int32)
        _check(lib().fir_lor_paths(self._h, C.byref(proj_desc(proj)), C.byref(vol_desc(vol, 1)), n,
                                   bins.ctypes.data, cap, coords.ctypes.data, lengths.ctypes.data,
                                   counts.ctypes.data, crosses.ctypes.data))
        return crosses, counts, coords, lengths


class Batch:
    """A ``fir_batch``: independent OSEM problems run together.

    problems: sequence of (ScannerSpec, ProjSpec, VolSpec, OSEMParams).
    """

    def __init__(self, ctx: Context, problems):
        self.ctx = ctx
        self.problems = list(problems)
        n = len(self.problems)
        sc = (ScannerDesc * n)(*[scanner_desc(p[0]) for p in self.problems])
        pr = (ProjDesc * n)(*[proj_desc(p[1]) for p in self.problems])
        vo = (VolDesc * n)(*[vol_desc(p[2], 1) for p in self.problems])
        pa = (OsemParamsDesc * n)(*[osem_desc(p[3]) for p in self.problems])
        self._h = C.c_void_p()
        _check(lib().fir_batch_create(C.byref(self._h), ctx.handle, n, sc, pr, vo, pa))

    def close(self) -> None:
        if self._h:
            lib().fir_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.problems)

    def set_data(self, p: int, sino, sens, bias=None) -> None:
        _, proj, vol, prm = self.problems[p]
        nb = proj_geometry(proj)["n_bins"]
        _check(lib().fir_batch_set_data(self._h, int(p), _ptr(sino, n=nb),
                                        _ptr(sens, n=vol.n_voxels * prm.n_subsets), _ptr(bias, n=nb)))

    def _n_voxels(self, p: int):
        # out-of-range indices are left to the library, which reports them
        return self.problems[p][2].n_voxels if 0 <= p < len(self.problems) else None

    def set_image(self, p: int, img) -> None:
        _check(lib().fir_batch_set_image(self._h, int(p), _ptr(img, n=self._n_voxels(p))))

    def get_image(self, p: int, img=None):
        vol = self.problems[p][2]
        if img is None:
            img = np.zeros(vol.shape_zyx, np.float32)
        _check(lib().fir_batch_get_image(self._h, int(p), _ptr(img, writable=True, n=vol.n_voxels)))
        return img

    def set_launch(self, block: int, blocks_per_sm: int, grab: int = 1) -> None:
        _check(lib().fir_batch_set_launch(self._h, int(block), int(blocks_per_sm), int(grab)))

    def launch(self):
        """(block, blocks_per_sm, grab) of the projector."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().fir_batch_get_launch(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def tune(self) -> float:
        ms = C.c_double()
        _check(lib().fir_batch_tune(self._h, C.byref(ms)))
        return ms.value

    def tune_report(self):
        """The last tune's candidates: [(block, blocks_per_sm, grab, axial_tile, ms), ...]."""
        n = C.c_int()
        _check(lib().fir_batch_tune_report(self._h, 0, None, None, None, None, None, C.byref(n)))
        k = n.value
        blk, per, grab, tile = (np.zeros(max(k, 1), np.int32) for _ in range(4))
        ms = np.zeros(max(k, 1), np.float64)
        _check(lib().fir_batch_tune_report(self._h, k, blk.ctypes.data, per.ctypes.data, grab.ctypes.data,
                                           tile.ctypes.data, ms.ctypes.data, C.byref(n)))
        return [(int(blk[i]), int(per[i]), int(grab[i]), int(tile[i]), float(ms[i])) for i in range(k)]

    def set_bundle(self, axial_tile: int) -> None:
        """Bundle shape: 0, 32 consecutive LORs; A in (1, 2, 4, 8), A axial
        planes x 32 / A tangential bins."""
        _check(lib().fir_batch_set_bundle(self._h, int(axial_tile)))

    def bundle(self) -> int:
        a = C.c_int()
        _check(lib().fir_batch_get_bundle(self._h, C.byref(a)))
        return a.value

    def schedule(self):
        """(steps, kernel launches) of the whole schedule."""
        n, k = C.c_int(), C.c_longlong()
        _check(lib().fir_batch_schedule(self._h, C.byref(n), C.byref(k)))
        return n.value, k.value

    def osem(self, use_graph: bool = True) -> None:
        _check(lib().fir_batch_osem(self._h, 1 if use_graph else 0))
