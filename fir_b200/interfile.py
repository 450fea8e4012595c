"""Interfile readers and writers for FIR's file formats, on the Python side.

Formats (all written by FIR's own writers, read by its KeyParser):

* scanner ``.scan`` -- ``!SCANNER PARAMETERS`` block
  (src_lib/ScannerInterfileReader.cc:6-52);
* sinogram ``.hs`` + raw little-endian float32 ``.s``, segments
  ``-so..+so`` concatenated, each ``[view][axial][tang]``
  (src_lib/ProjInterfileReader.cc:13-192);
* volume ``.h33`` + ``.i33`` (src_lib/VolInterfileReader.cc:137-661); reads
  every number format FIR reads (unsigned/signed integers of 1, 2, 4, 8 bytes,
  float of 4 or 8 bytes, either byte order), writes FLOAT 4 LITTLEENDIAN;
* parameter files of the three executables (keys of src_bin/*.cc).

Keywords follow Interfile 3.3 conventions as implemented by
``KeyParser::standardiseKeyword`` (src_lib/KeyParser.cc:589-651): space, tab,
``_`` and ``!`` are white space, runs of white space collapse, case is
ignored; ``${ENV}`` is substituted (:426-465) and ``{a, b}`` is a list.
"""
from __future__ import annotations

import os
import re
from typing import Dict, Optional, Tuple

import numpy as np

from .geometry import ProjSpec, ScannerSpec, VolSpec

__all__ = [
    "standardise_keyword",
    "parse_keys",
    "write_scanner",
    "read_scanner",
    "write_proj",
    "write_proj_header",
    "read_proj_header",
    "read_proj",
    "write_vol",
    "write_vol_header",
    "read_vol",
]


def standardise_keyword(kw: str) -> str:
    out = []
    prev_ws = False
    s = kw.strip(" \t_!")
    for ch in s:
        if ch.isspace() or ch in "_!":
            if not prev_ws:
                out.append(" ")
                prev_ws = True
        else:
            if ch == "[" and not prev_ws:
                out.append(" [")
            else:
                out.append(ch.lower())
            prev_ws = False
    return "".join(out)


_ENV = re.compile(r"\$\{([^}]*)\}")


def parse_keys(path: str, start_key: str, stop_key: Optional[str] = None) -> Dict[str, str]:
    """Raw ``key -> value`` strings between ``start_key`` and ``stop_key``."""
    start = standardise_keyword(start_key)
    stop = standardise_keyword(stop_key) if stop_key else "end of " + start
    with open(path, "r") as f:
        lines = f.read().splitlines()
    out: Dict[str, str] = {}
    parsing = False
    for line in lines:
        if not line.strip(" \t"):
            continue
        line = _ENV.sub(lambda m: os.environ.get(m.group(1), ""), line)
        key = standardise_keyword(line.split(":", 1)[0])
        if not parsing:
            if key == start:
                parsing = True
                continue
            raise ValueError(f'{path}: required first keyword "{start}" not found')
        if key == stop:
            return out
        value = ""
        if "=" in line:
            value = line.split("=", 1)[1].strip(" \t")
        out[key] = value
    return out


def _list(v: str, conv):
    v = v.strip()
    if v.startswith("{"):
        inner = v[1 : v.index("}")] if "}" in v else v[1:]
        return [conv(x) for x in inner.split(",") if x.strip()]
    return [conv(v.split()[0])]


def _fmt_list(vals) -> str:
    return "{" + ", ".join(repr(float(x)) if isinstance(x, float) else str(x) for x in vals) + "}"


def _fmt_double(x: float) -> str:
    # writeKeys.cc:12-21 writes doubles with "%.7f"
    return "%.7f" % float(x)


# ---------------------------------------------------------------- scanner

def write_scanner(path: str, s: ScannerSpec) -> None:
    lines = [
        "!SCANNER PARAMETERS :=",
        f"crystal dimensions XYZ in mm := {_fmt_list([float(x) for x in s.crystal_dims])}",
        f"crystal repeat numbers YZ := {_fmt_list([int(x) for x in s.crystal_repeat])}",
        f"inter-crystal distance YZ in mm := {_fmt_list([float(x) for x in s.inter_crystal])}",
        f"module dimensions XYZ in mm := {_fmt_list([float(x) for x in s.module_dims])}",
        f"module repeat numbers YZ := {_fmt_list([int(x) for x in s.module_repeat])}",
        f"inter-module distance YZ in mm := {_fmt_list([float(x) for x in s.inter_module])}",
        f"rSector dimensions XYZ in mm := {_fmt_list([float(x) for x in s.rsector_dims])}",
        f"rSector repeat number := {int(s.rsector_repeat_number)}",
        f"rSector inner radius in mm := {repr(float(s.rsector_inner_radius))}",
        "!END OF SCANNER PARAMETERS :=",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_scanner(path: str) -> ScannerSpec:
    k = parse_keys(path, "!SCANNER PARAMETERS", "!END OF SCANNER PARAMETERS")

    def get(key, conv, n, default):
        return tuple(_list(k[key], conv)) if k.get(key) else tuple([default] * n)

    return ScannerSpec(
        rsector_repeat_number=int(k.get("rsector repeat number", "0") or 0),
        rsector_inner_radius=float(k.get("rsector inner radius in mm", "0") or 0),
        crystal_dims=get("crystal dimensions xyz in mm", float, 3, 0.0),
        crystal_repeat=get("crystal repeat numbers yz", int, 2, 1),
        inter_crystal=get("inter-crystal distance yz in mm", float, 2, 0.0),
        module_dims=get("module dimensions xyz in mm", float, 3, 0.0),
        module_repeat=get("module repeat numbers yz", int, 2, 1),
        inter_module=get("inter-module distance yz in mm", float, 2, 0.0),
        rsector_dims=get("rsector dimensions xyz in mm", float, 3, 0.0),
    )


# -------------------------------------------------------------- sinograms

def write_proj_header(path: str, p: ProjSpec, data_file: str = "") -> None:
    lines = [
        "!PROJECTION DATA PARAMETERS :=",
        f"name of data file := {data_file}",
        f"number of rings := {p.n_rings}",
        f"number of crystals per ring := {p.n_crystals_per_ring}",
        f"segment span := {p.segment_span}",
        f"number of segments := {p.n_segments}",
        f"number of tangential coordinates := {p.n_tang_coords}",
        "!END OF PROJECTION DATA PARAMETERS :=",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_proj(base: str, p: ProjSpec, data: np.ndarray) -> str:
    """Writes ``base.hs`` and ``base.s``; returns the header path."""
    root = os.path.splitext(base)[0]
    hs, s = root + ".hs", root + ".s"
    write_proj_header(hs, p, os.path.basename(s))
    np.ascontiguousarray(data, dtype="<f4").tofile(s)
    return hs


def read_proj_header(path: str) -> Tuple[ProjSpec, str]:
    k = parse_keys(path, "!PROJECTION DATA PARAMETERS", "!END OF PROJECTION DATA PARAMETERS")

    def gi(key, default):
        v = k.get(key, "")
        return int(v.split()[0]) if v.strip() else default

    spec = ProjSpec(
        n_rings=gi("number of rings", 0),
        n_crystals_per_ring=gi("number of crystals per ring", 0),
        segment_span=gi("segment span", 1),
        n_segments=gi("number of segments", 1),
        n_tang_coords=gi("number of tangential coordinates", 0),
    )
    data = k.get("name of data file", "")
    if data and not data.startswith("/"):
        data = os.path.join(os.path.dirname(path), data)
    return spec, data


def read_proj(path: str, n_bins: int) -> Tuple[ProjSpec, np.ndarray]:
    spec, data = read_proj_header(path)
    arr = np.fromfile(data, dtype="<f4")
    if arr.size < n_bins:
        raise ValueError(
            f"The number of bins that were read from the data file ({arr.size}) is inferior "
            f"to that expected from the header file ({n_bins})"
        )
    return spec, arr[:n_bins].astype(np.float32)


# ---------------------------------------------------------------- volumes

def write_vol_header(path: str, v: VolSpec, data_file: str = "") -> None:
    lines = [
        "!INTERFILE :=",
        "",
        f"name of data file := {data_file}",
        "data offset in bytes := 0",
        "number format := FLOAT",
        "number of bytes per pixel := 4",
        "imagedata byte order := LITTLEENDIAN",
        "",
        "number of dimensions := 3",
        "",
        f"matrix size [1] := {int(v.size[0])}",
        f"matrix size [2] := {int(v.size[1])}",
        f"matrix size [3] := {int(v.size[2])}",
        f"number of slices := {int(v.size[2])}",
        "",
        f"scaling factor (mm/pixel) [1] := {_fmt_double(v.voxel[0])}",
        f"scaling factor (mm/pixel) [2] := {_fmt_double(v.voxel[1])}",
        f"scaling factor (mm/pixel) [3] := {_fmt_double(v.voxel[2])}",
        f"slice thickness (pixels) := {_fmt_double(v.voxel[2])}",
        "",
        f"first pixel offset (mm) [1] := {_fmt_double(v.offset[0])}",
        f"first pixel offset (mm) [2] := {_fmt_double(v.offset[1])}",
        f"first pixel offset (mm) [3] := {_fmt_double(v.offset[2])}",
        "",
        f"number of time frames := {int(v.n_frames)}",
        "",
        "!END OF INTERFILE :=",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_vol(base: str, v: VolSpec, data: np.ndarray) -> str:
    """Writes ``base.h33`` and ``base.i33`` (FLOAT 4 LITTLEENDIAN)."""
    root = os.path.splitext(base)[0]
    h, d = root + ".h33", root + ".i33"
    write_vol_header(h, v, os.path.basename(d))
    np.ascontiguousarray(data, dtype="<f4").tofile(d)
    return h


_NUMBER_FORMATS = {
    ("SHORT FLOAT", 4): "f4",
    ("LONG FLOAT", 8): "f8",
    ("FLOAT", 4): "f4",
    ("FLOAT", 8): "f8",
}


def read_vol(path: str, read_data: bool = True):
    """Returns ``(VolSpec, data or None)``; data is float32 ``[frames*nz, ny, nx]``."""
    k = parse_keys(path, "!INTERFILE", "!END OF INTERFILE")

    def g(key, conv, default):
        v = k.get(key, "")
        return conv(v.split()[0]) if v.strip() else default

    size = (g("matrix size [1]", int, 0), g("matrix size [2]", int, 0), g("number of slices", int, 0))
    voxel = (
        g("scaling factor (mm/pixel) [1]", float, 0.0),
        g("scaling factor (mm/pixel) [2]", float, 0.0),
        g("slice thickness (pixels)", float, 0.0),
    )
    offset = (
        g("first pixel offset (mm) [1]", float, 0.0),
        g("first pixel offset (mm) [2]", float, 0.0),
        g("first pixel offset (mm) [3]", float, 0.0),
    )
    spec = VolSpec(size, voxel, offset, g("number of time frames", int, 1))
    if min(size) <= 0:
        raise ValueError("Number of voxels must be greater than zero in each dimension")
    if min(voxel) <= 0:
        raise ValueError("Voxel extent must be greater than zero in each dimension")
    data_file = k.get("name of data file", "")
    if not read_data or not data_file:
        return spec, None
    if not data_file.startswith("/"):
        data_file = os.path.join(os.path.dirname(path), data_file)
    fmt = k.get("number format", "").upper()
    nbytes = g("number of bytes per pixel", int, 0)
    order = k.get("imagedata byte order", "").upper() or "LITTLEENDIAN"
    if fmt in ("UNSIGNED INTEGER", "SIGNED INTEGER"):
        nbytes = nbytes if nbytes in (1, 2, 4, 8) else 4
        code = ("u" if fmt.startswith("UNSIGNED") else "i") + str(nbytes)
    elif (fmt, nbytes) in _NUMBER_FORMATS:
        code = _NUMBER_FORMATS[(fmt, nbytes)]
    elif fmt in ("SHORT FLOAT", "FLOAT"):
        code = "f4"
    elif fmt == "LONG FLOAT":
        code = "f8"
    else:
        raise ValueError(f"Unrecognized data type name {fmt}")
    dt = np.dtype(("<" if order == "LITTLEENDIAN" else ">") + code)
    n = spec.n_voxels * spec.n_frames
    off = g("data offset in bytes", int, 0)
    raw = np.fromfile(data_file, dtype=dt, count=n, offset=off)
    if raw.size < n:
        raise ValueError(
            f"The number of pixels that were read from the data file ({raw.size}) is inferior "
            f"to the number expected from the header file ({n})"
        )
    data = raw.astype(np.float32).reshape(spec.n_frames * size[2], size[1], size[0])
    return spec, data
