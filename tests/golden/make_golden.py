"""Generates the committed golden fixtures of tests/golden/ by running FIR's
own compiled code (oracle/_ref/libfirref.so, built from the FIR sources by
oracle/Makefile) on small seeded inputs.

    python tests/golden/make_golden.py

Fixtures:
  siddon_cases.npz   -- Siddon paths of FIR's unit-test geometries
                        (src_test/SiddonUnitTest.cc: a 3x3x2 volume of
                        1x2x3 mm voxels and a 512x384x1 volume of 1x2x1 mm
                        voxels) for the segment families those tests use --
                        misses along the borders, rows, columns and z-lines
                        through every voxel, segments starting or stopping
                        at a voxel centre -- plus seeded random segments.
  proj_geometry.json -- ProjGeometry of FIR's unit-test headers
                        (src_test/ProjHeaderUnitTest.cc:181-232) and of the
                        benchmark sinograms.
  tiny_ref.npz       -- forward projection, 4-subset backprojection,
                        sensitivity and a 2x4 OSEM run with Gaussian filter of
                        the seeded "tiny" workload, all by FIR (1 thread).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fir_b200 import workloads  # noqa: E402
from fir_b200.geometry import OSEMParams, ProjSpec, VolSpec  # noqa: E402
from oracle import bridge  # noqa: E402


def unit_geometries():
    """The two volumes of FIR's Siddon unit tests, centred in x and y."""
    small = VolSpec.centred((3, 3, 2), (1.0, 2.0, 3.0))
    long = VolSpec.centred((512, 384, 1), (1.0, 2.0, 1.0))
    return small, long


def family_segments(v: VolSpec):
    """Segments of the kinds FIR's unit tests exercise, for every row,
    column and z-line of the volume (vectorised over the volume)."""
    nx, ny, nz = (int(s) for s in v.size)
    vx, vy, vz = (float(s) for s in v.voxel)
    x, y, z = v.voxel_centres()
    # planes one voxel outside the volume on each side
    left, right = x[0] - vx, x[0] - vx + (nx + 1) * vx
    top, bottom = y[0] - vy, y[0] - vy + (ny + 1) * vy
    front, back = z[0] - vz, z[-1] + vz
    segs = []
    # misses: along the four outer lines of slice 0
    segs += [(left, top, z[0], right, top, z[0]), (left, bottom, z[0], right, bottom, z[0]),
             (left, top, z[0], left, bottom, z[0]), (right, top, z[0], right, bottom, z[0])]
    for k in range(nz):
        for j in range(min(ny, 8)):
            segs.append((left, y[j], z[k], right, y[j], z[k]))      # rows
        for i in range(min(nx, 8)):
            segs.append((x[i], top, z[k], x[i], bottom, z[k]))      # columns
    for j in range(min(ny, 4)):
        for i in range(min(nx, 4)):
            segs.append((x[i], y[j], front, x[i], y[j], back))      # z-lines
    # starting inside (at a voxel centre) and going backwards, and stopping inside
    segs.append((x[nx // 2], y[0], z[0], left, y[0], z[0]))
    segs.append((x[0], y[ny // 2], z[0], x[0], top, z[0]))
    segs.append((x[0], y[0], z[-1], x[0], y[0], front))
    segs.append((right, y[0], z[0], x[nx // 2], y[0], z[0]))
    segs.append((x[0], bottom, z[0], x[0], y[ny // 2], z[0]))
    segs.append((x[0], y[0], back, x[0], y[0], z[0]))
    return np.array(segs, np.float64)


def random_segments(v: VolSpec, n: int, seed: int):
    rng = np.random.default_rng(seed)
    ext = np.array([v.size[i] * v.voxel[i] for i in range(3)])
    c = np.array([v.offset[0] + (v.size[0] - 1) * v.voxel[0] / 2,
                  v.offset[1] + (v.size[1] - 1) * v.voxel[1] / 2, v.offset[2]])
    a = c + rng.uniform(-1.0, 1.0, (n, 3)) * ext
    b = c + rng.uniform(-1.0, 1.0, (n, 3)) * ext
    # a share of axis-parallel and plane-parallel segments (cancelled dims)
    k = n // 4
    b[:k, 2] = a[:k, 2]
    b[k:2 * k, 1] = a[k:2 * k, 1]
    return np.concatenate([a, b], axis=1)


def main():
    bridge.build(reference=True)
    ref = bridge.Reference()
    ref.threads(1)

    out = {}
    for name, v in zip(("unit3x3x2", "unit512x384"), unit_geometries()):
        segs = np.concatenate([family_segments(v), random_segments(v, 200, 7)])
        crosses, counts, coords, lengths = ref.siddon_paths(v, segs)
        out[name + "_vol"] = np.array(list(v.size) + list(v.voxel) + list(v.offset), np.float64)
        out[name + "_segs"] = segs
        out[name + "_crosses"] = crosses
        out[name + "_counts"] = counts
        out[name + "_coords"] = coords
        out[name + "_lengths"] = lengths
    np.savez_compressed(os.path.join(HERE, "siddon_cases.npz"), **out)

    geo = {}
    cases = {
        "span1_5x32": ProjSpec(5, 32, 3, 8, 1),
        "span3_5x32": ProjSpec(5, 32, 3, 8, 3),
        "demo_39x624": ProjSpec(39, 624, 3, 380, 3),
        "small": workloads.small().proj,
        "clinical": workloads.clinical().proj,
        "clinical_fullfov": workloads.clinical(full_fov=True).proj,
        "large": workloads.large().proj,
    }
    for k, p in cases.items():
        d = ref.proj_geometry(p)
        d["header"] = [p.n_rings, p.n_crystals_per_ring, p.n_segments, p.n_tang_coords, p.segment_span]
        geo[k] = d
    with open(os.path.join(HERE, "proj_geometry.json"), "w") as f:
        json.dump(geo, f, indent=1, sort_keys=True)

    w = workloads.tiny()
    x = workloads.activity(w)
    sino = ref.forward(w.scanner, w.proj, w.vol, x, ref.proj_geometry(w.proj)["n_bins"])
    bp4 = ref.backward(w.scanner, w.proj, w.vol.with_frames(4), sino, 4)
    sens = ref.sensitivity(w.scanner, w.proj, w.vol.with_frames(4), 4)
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0])
    y = workloads.poisson_counts(sino, w.counts, w.seed)
    osem = ref.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm)
    np.savez_compressed(os.path.join(HERE, "tiny_ref.npz"), image=x, sino=sino, bp4=bp4, sens4=sens, counts=y,
                        osem=osem)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
