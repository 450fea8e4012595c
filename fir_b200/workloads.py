"""Seeded synthetic workloads: scanners, sinogram headers, volumes, phantoms.

FIR publishes no benchmark data, so every measurement and parity case runs on
seeded synthetic phantoms with the shapes, sizes and value ranges of the
benchmark configurations:

* ``small``    -- 8 rings x 128 crystals, R = 200 mm, LORs within 100 mm of
                  the axis; 64x64x16 image at 4 mm; cylinder + 2 hot spheres;
                  water attenuation; 1e6 counts; OSEM 4 subsets x 3 iterations,
                  FWHM 4 mm.
* ``clinical`` -- 32 rings x 512 crystals, R = 400 mm, LORs within 150 mm of
                  the axis (3.28e7 LORs; ``full_fov=True`` gives all 511
                  tangential bins, 1.34e8 LORs); 200x200x64 image at 3 mm;
                  elliptical water body with 10 ellipsoids; 5e8 counts; OSEM 16
                  subsets x 2 iterations, FWHM 4 mm.
* ``large``    -- 64 rings x 640 crystals, R = 410 mm, ring pitch 3.2 mm, LORs
                  within 160 mm; 320x320x128 image at 1.5 mm (exact geometry);
                  40 ellipsoids + 20 hot spheres; 2e9 counts; 28 subsets x 1.
* ``batched``  -- 64 small problems of uneven sizes (``batch_problems``).
* ``autograd`` -- the clinical scanner with 8 ellipsoid phantoms on a
                  128x128x48 image at 3 mm (``autograd_batch``).

The phantom arrays are float32 ``[nz, ny, nx]``.  Measured data are made by
the caller's forward projector: ``expected = scale * A x / ACF`` with the
attenuation correction factors ``ACF = exp(A mu)``, then Poisson-sampled.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .geometry import OSEMParams, ProjSpec, ScannerSpec, VolSpec

GEOMETRY_REFERENCE = 0
GEOMETRY_EXACT = 1


def n_tang_for_fov(n_crystals: int, radius: float, fov_radius: float) -> int:
    """Tangential bins whose LOR passes within ``fov_radius`` of the axis.

    Bin t of a view is the chord between crystals whose angular distance is
    pi - 2*pi*|t|/(2N)..., i.e. at distance R*sin(pi*|t|/N) from the axis.
    """
    tmax = int(math.floor(n_crystals / math.pi * math.asin(min(1.0, fov_radius / radius))))
    return 2 * tmax + 1


@dataclass
class Workload:
    name: str
    scanner: ScannerSpec
    proj: ProjSpec
    vol: VolSpec
    osem: OSEMParams
    counts: float
    seed: int
    geometry: int = GEOMETRY_REFERENCE
    kind: str = "cylinder"  # phantom family
    extra: dict = field(default_factory=dict)

    @property
    def n_lors(self) -> int:
        from .capi import proj_geometry

        return proj_geometry(self.proj)["n_bins"]


def small(seed: int = 1) -> Workload:
    n_rings, n_cpr, radius = 8, 128, 200.0
    return Workload(
        name="small",
        scanner=ScannerSpec.ring(n_rings, n_cpr, radius, 4.0),
        proj=ProjSpec(n_rings, n_cpr, 2 * n_rings - 1, n_tang_for_fov(n_cpr, radius, 100.0)),
        vol=VolSpec((64, 64, 16), (4.0, 4.0, 4.0), (-126.0, -126.0, 0.0)),
        osem=OSEMParams(n_iterations=3, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
        counts=1e6,
        seed=seed,
        kind="cylinder",
    )


def clinical(seed: int = 2, full_fov: bool = False) -> Workload:
    n_rings, n_cpr, radius = 32, 512, 400.0
    n_tang = n_cpr - 1 if full_fov else n_tang_for_fov(n_cpr, radius, 150.0)
    return Workload(
        name="clinical" + ("-fullfov" if full_fov else ""),
        scanner=ScannerSpec.ring(n_rings, n_cpr, radius, 4.0),
        proj=ProjSpec(n_rings, n_cpr, 2 * n_rings - 1, n_tang),
        vol=VolSpec((200, 200, 64), (3.0, 3.0, 3.0), (-298.5, -298.5, 0.0)),
        osem=OSEMParams(n_iterations=2, n_subsets=16, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
        counts=5e8,
        seed=seed,
        kind="body",
        extra={"body": (150.0, 110.0), "n_ellipsoids": 10},
    )


def large(seed: int = 5) -> Workload:
    n_rings, n_cpr, radius = 64, 640, 410.0
    return Workload(
        name="large",
        scanner=ScannerSpec.ring(n_rings, n_cpr, radius, 3.2),
        proj=ProjSpec(n_rings, n_cpr, 2 * n_rings - 1, n_tang_for_fov(n_cpr, radius, 160.0)),
        vol=VolSpec.centred((320, 320, 128), (1.5, 1.5, 1.5)),
        osem=OSEMParams(n_iterations=1, n_subsets=28 if (n_cpr // 2) % 28 == 0 else 32,
                        convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
        counts=2e9,
        seed=seed,
        geometry=GEOMETRY_EXACT,
        kind="body",
        extra={"body": (155.0, 115.0), "n_ellipsoids": 40, "n_spheres": 20},
    )


def autograd_batch(n: int = 8, seed: int = 11) -> List[Workload]:
    """The differentiable-projector workload: the clinical scanner and
    field of view, ``n`` seeded ellipsoid phantoms (elliptical water body with
    10 ellipsoids) on a 128x128x48 image at 3 mm, 5e8 counts each."""
    base = clinical()
    rng = np.random.default_rng(seed)
    return [Workload(
        name=f"autograd{i}",
        scanner=base.scanner,
        proj=base.proj,
        vol=VolSpec.centred((128, 128, 48), (3.0, 3.0, 3.0)),
        osem=base.osem,
        counts=5e8,
        seed=int(rng.integers(1 << 30)),
        kind="body",
        extra={"body": (150.0, 110.0), "n_ellipsoids": 10},
    ) for i in range(n)]


def tiny(seed: int = 0) -> Workload:
    """A few-thousand-LOR case for smoke tests and the CPU suite."""
    n_rings, n_cpr, radius = 4, 64, 120.0
    return Workload(
        name="tiny",
        scanner=ScannerSpec.ring(n_rings, n_cpr, radius, 4.0),
        proj=ProjSpec(n_rings, n_cpr, 2 * n_rings - 1, n_tang_for_fov(n_cpr, radius, 60.0)),
        vol=VolSpec((32, 32, 8), (4.0, 4.0, 4.0), (-62.0, -62.0, 0.0)),
        osem=OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
        counts=1e5,
        seed=seed,
        kind="cylinder",
    )


def batch_problems(n: int = 64, seed: int = 3) -> List[Workload]:
    """Uneven reconstructions: 4-24 rings x 96-384 crystals (multiples of 4),
    radius 150-400 mm, images 32^2x8 .. 128^2x48 at 2-4 mm, 1e5-1e7 counts
    (log-uniform), 4-12 subsets dividing the number of views, 3 iterations."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        n_rings = int(rng.integers(4, 25))
        # crystals: a multiple of 4 whose number of views has a divisor in [4, 12]
        divisors = []
        while not divisors:
            n_cpr = 4 * int(rng.integers(24, 97))
            divisors = [d for d in range(4, 13) if (n_cpr // 2) % d == 0]
        radius = float(rng.uniform(150.0, 400.0))
        vox = float(rng.choice([2.0, 3.0, 4.0]))
        nxy = int(rng.integers(32, 129))
        nz = int(rng.integers(8, 49))
        n_sub = int(rng.choice(divisors))
        half_width = nxy * vox / 2.0
        fov = min(0.9 * half_width, 0.7 * radius)
        out.append(Workload(
            name=f"batch{i}",
            scanner=ScannerSpec.ring(n_rings, n_cpr, radius, 4.0),
            proj=ProjSpec(n_rings, n_cpr, 2 * n_rings - 1, n_tang_for_fov(n_cpr, radius, fov)),
            vol=VolSpec.centred((nxy, nxy, nz), (vox, vox, vox)),
            osem=OSEMParams(n_iterations=3, n_subsets=n_sub, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0]),
            counts=float(10 ** rng.uniform(5, 7)),
            seed=int(rng.integers(1 << 30)),
            kind="cylinder",
            extra={"cyl_radius": 0.7 * fov},
        ))
    return out


# ------------------------------------------------------------- phantoms

def _grid(v: VolSpec):
    x, y, z = v.voxel_centres()
    return np.meshgrid(z, y, x, indexing="ij")  # Z, Y, X each [nz, ny, nx]


def activity(w: Workload) -> np.ndarray:
    """Seeded activity phantom of the workload, float32 [nz, ny, nx]."""
    rng = np.random.default_rng(w.seed)
    Z, Y, X = _grid(w.vol)
    img = np.zeros(Z.shape, np.float32)
    if w.kind == "cylinder":
        r = w.extra.get("cyl_radius", 80.0)
        inside = X ** 2 + Y ** 2 <= r ** 2
        img[inside] = 1.0
        half_depth = w.vol.size[2] * w.vol.voxel[2] / 2.0
        for _ in range(2):
            rad = 10.0 if r >= 40 else r / 4
            rho = rng.uniform(0, r - rad)
            phi = rng.uniform(0, 2 * math.pi)
            cz = rng.uniform(-max(0.0, half_depth - rad), max(0.0, half_depth - rad))
            cx, cy = rho * math.cos(phi), rho * math.sin(phi)
            img[(X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2 <= rad ** 2] = 4.0
        return img
    a, b = w.extra["body"]
    body = (X / a) ** 2 + (Y / b) ** 2 <= 1.0
    img[body] = 1.0
    for _ in range(int(w.extra.get("n_ellipsoids", 10))):
        sa = rng.uniform(10.0, 120.0, size=3)
        theta = rng.uniform(0, math.pi)
        u = rng.uniform(-0.7, 0.7, size=2)
        cx, cy = u[0] * a, u[1] * b
        cz = rng.uniform(-0.5, 0.5) * w.vol.size[2] * w.vol.voxel[2] / 2
        ct, st = math.cos(theta), math.sin(theta)
        xr = (X - cx) * ct + (Y - cy) * st
        yr = -(X - cx) * st + (Y - cy) * ct
        m = (xr / sa[0]) ** 2 + (yr / sa[1]) ** 2 + ((Z - cz) / sa[2]) ** 2 <= 1.0
        img[m & body] = rng.uniform(0.5, 5.0)
    for _ in range(int(w.extra.get("n_spheres", 0))):
        rad = rng.uniform(2.0, 8.0)
        u = rng.uniform(-0.7, 0.7, size=2)
        cx, cy = u[0] * a, u[1] * b
        cz = rng.uniform(-0.5, 0.5) * w.vol.size[2] * w.vol.voxel[2] / 2
        img[((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2 <= rad ** 2) & body] = 8.0
    return img


def hounsfield(w: Workload) -> np.ndarray:
    """Attenuation map in Hounsfield units: water (0 HU) inside the body or
    cylinder, air (-1000 HU) outside; FIR converts it to mu = 0.0096/mm."""
    Z, Y, X = _grid(w.vol)
    if w.kind == "cylinder":
        r = w.extra.get("cyl_radius", 80.0)
        inside = X ** 2 + Y ** 2 <= r ** 2
    else:
        a, b = w.extra["body"]
        inside = (X / a) ** 2 + (Y / b) ** 2 <= 1.0
    return np.where(inside, 0.0, -1000.0).astype(np.float32)


def poisson_counts(expected: np.ndarray, total: float, seed: int) -> np.ndarray:
    """Scales ``expected`` to ``total`` counts and draws Poisson samples."""
    s = float(expected.sum(dtype=np.float64))
    lam = expected.astype(np.float64) * (total / s if s > 0 else 0.0)
    return np.random.default_rng(seed).poisson(lam).astype(np.float32)


def measured_sinogram(w: Workload, ax: np.ndarray, line_mu: Optional[np.ndarray]) -> np.ndarray:
    """Measured, attenuation-precorrected data of ``w`` from two forward
    projections made by the caller's projector: ``ax`` = A x of the phantom
    and ``line_mu`` = A mu of the attenuation map (FIR's HU-to-mu map), both
    float32 in FIR's file order; ``line_mu=None`` means no attenuation.

    The attenuation correction factors are ACF = exp(A mu) where A mu > 1e-5,
    else 1 (ProjData::exponential, ProjData.cc:514-539; evaluated in double
    and rounded once).  The expected counts A x / ACF are scaled to
    ``w.counts``, Poisson-sampled with ``w.seed`` and multiplied by the
    factors again, zero where either operand is <= 1e-5 (ProjData::operator*=,
    ProjData.cc:481-512; the OSEM executable's precorrection, OSEM.cc:294-337).
    Everything after the two projections runs here in numpy, so projectors
    whose forward projections agree bit for bit (this library's and FIR's
    own) give bit-identical data."""
    ax = np.ascontiguousarray(ax, np.float32)
    if line_mu is None:
        acf = np.ones_like(ax)
    else:
        lm = np.ascontiguousarray(line_mu, np.float32)
        acf = np.where(lm.astype(np.float64) > 1e-5, np.exp(lm.astype(np.float64)), 1.0).astype(np.float32)
    expected = ax / acf
    s = float(expected.sum(dtype=np.float64))
    expected *= np.float32(w.counts / s if s > 0 else 0.0)
    y = np.random.default_rng(w.seed).poisson(expected.astype(np.float64)).astype(np.float32)
    keep = (y.astype(np.float64) > 1e-5) & (acf.astype(np.float64) > 1e-5)
    return np.where(keep, y * acf, np.float32(0.0)).astype(np.float32)


def measured_on_gpu(ctx, w: Workload, device, attenuation: bool = True):
    """Measured data of ``w`` made with the GPU projector of ``ctx`` (scanner
    and geometry already set): the phantom is forward-projected, divided by
    the attenuation factors exp(A mu) when ``attenuation``, scaled to
    ``w.counts``, Poisson-sampled with ``w.seed`` and precorrected by the
    factors again (OSEM.cc:294-337).  Returns (sinogram, sensitivity with
    ``w.osem.n_subsets`` frames) as device tensors."""
    import torch

    nb = w.n_lors
    x_true = torch.from_numpy(activity(w)).to(device)
    ax = torch.empty(nb, device=device)
    ctx.forward(w.vol, x_true, w.proj, ax)
    acf = None
    if attenuation:
        mu = torch.from_numpy(hounsfield(w)).to(device)
        ctx.hu_to_mu(w.vol, mu)
        acf = torch.empty(nb, device=device)
        ctx.forward_exp(w.vol, mu, w.proj, acf)
        ax = ax / acf
    ax *= w.counts / float(ax.sum(dtype=torch.float64))
    gen = torch.Generator(device=device).manual_seed(w.seed)
    y = torch.poisson(ax, generator=gen)
    if acf is not None:
        ctx.proj_multiply(w.proj, y, acf)
    nsub = w.osem.n_subsets
    sens = torch.empty((nsub,) + tuple(w.vol.shape_zyx), device=device)
    ctx.sensitivity(w.proj, w.vol, sens, nsub)
    return y, sens
