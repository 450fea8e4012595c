"""Geometry descriptors of the FIR data model, mirrored on the Python side.

They carry the same fields as FIR's headers and are converted to the C-ABI
descriptors of ``include/fir_cuda.h`` by :mod:`fir_b200.capi`:

* :class:`ScannerSpec` -- ``ScannerHeader`` (src_lib/ScannerHeader.h:7-46)
* :class:`ProjSpec`    -- ``ProjHeader`` (src_lib/ProjHeader.h:15-40)
* :class:`VolSpec`     -- ``VolHeader`` (src_lib/VolHeader.h:7-23)

Derived quantities (``ProjGeometry::fill``, ``ScannerData`` position tables)
are computed by the native library, never re-derived here, so that Python and
C++ callers see bit-identical tables.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import List, Sequence


@dataclass
class ScannerSpec:
    """Cylindrical scanner built from crystals, modules and rSectors.

    Zero dimensions mean "fit tightly on the level below" and zero repeat
    numbers are invalid, as in ``ScannerHeader::check`` (ScannerHeader.cc:26-303).
    """

    rsector_repeat_number: int
    rsector_inner_radius: float
    crystal_dims: Sequence[float] = (0.0, 0.0, 0.0)
    crystal_repeat: Sequence[int] = (1, 1)
    inter_crystal: Sequence[float] = (0.0, 0.0)
    module_dims: Sequence[float] = (0.0, 0.0, 0.0)
    module_repeat: Sequence[int] = (1, 1)
    inter_module: Sequence[float] = (0.0, 0.0)
    rsector_dims: Sequence[float] = (0.0, 0.0, 0.0)

    @property
    def n_crystals_per_ring(self) -> int:
        return int(self.crystal_repeat[0] * self.module_repeat[0] * self.rsector_repeat_number)

    @property
    def n_rings(self) -> int:
        return int(self.crystal_repeat[1] * self.module_repeat[1])

    @classmethod
    def ring(cls, n_rings: int, n_crystals: int, radius: float, ring_pitch: float) -> "ScannerSpec":
        """A ring scanner with point crystals evenly spaced in angle:
        one crystal per rSector, ``n_rings`` crystals of depth ``ring_pitch``
        stacked along z (crystal centres on a circle of ``radius``)."""
        return cls(
            rsector_repeat_number=n_crystals,
            rsector_inner_radius=radius,
            crystal_dims=(0.0, 0.0, ring_pitch),
            crystal_repeat=(1, n_rings),
        )


@dataclass
class ProjSpec:
    """Sinogram header.  ``n_tang_coords = 0`` selects the maximum
    (``n_crystals_per_ring - 1``), as ``ProjHeader::check`` does."""

    n_rings: int
    n_crystals_per_ring: int
    n_segments: int = 1
    n_tang_coords: int = 0
    segment_span: int = 1


@dataclass
class VolSpec:
    """Volume header: voxel counts, voxel extents (mm) and offsets.

    ``offset[0:2]`` is the centre of the first voxel in x and y;
    ``offset[2]`` is the z offset of the volume centre from the scanner centre
    (VolHeader.h:14-17).
    """

    size: Sequence[int]
    voxel: Sequence[float]
    offset: Sequence[float] = (0.0, 0.0, 0.0)
    n_frames: int = 1

    @property
    def n_voxels(self) -> int:
        return int(self.size[0]) * int(self.size[1]) * int(self.size[2])

    @property
    def shape_zyx(self):
        return (int(self.size[2]), int(self.size[1]), int(self.size[0]))

    def with_frames(self, n: int) -> "VolSpec":
        return replace(self, n_frames=n)

    @classmethod
    def centred(cls, size: Sequence[int], voxel: Sequence[float], z_offset: float = 0.0) -> "VolSpec":
        """A volume centred on the scanner axis."""
        ox = -(size[0] - 1) * voxel[0] / 2.0
        oy = -(size[1] - 1) * voxel[1] / 2.0
        return cls(tuple(size), tuple(voxel), (ox, oy, z_offset))

    def voxel_centres(self):
        """(x[i], y[j], z[k]) centre coordinates in mm, as numpy arrays."""
        import numpy as np

        nx, ny, nz = (int(s) for s in self.size)
        vx, vy, vz = (float(v) for v in self.voxel)
        x = self.offset[0] + vx * np.arange(nx)
        y = self.offset[1] + vy * np.arange(ny)
        z = self.offset[2] - nz * vz / 2.0 + vz * (np.arange(nz) + 0.5)
        return x, y, z


@dataclass
class OSEMParams:
    """``OSEMCoreParams`` (src_lib/reconAlgos.h:9-22)."""

    n_iterations: int = 1
    n_subsets: int = 1
    save_interval: int = 0
    cut_radius: float = 0.0
    convolution_interval: int = 0
    fwhm_xyz: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
