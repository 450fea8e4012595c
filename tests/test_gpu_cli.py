"""The drop-in executables against FIR's own, on the same files.

Three builds of each program run on identical inputs:
- ours (fir_b200/bin/FIR_*);
- FIR's, compiled from its sources (oracle/_ref/FIR_*, one OpenMP thread so its float
  atomics sum in LOR order);
- FIR's unmodified sources compiled against our drop-in headers and libraries
  (oracle/_ref/dropin/FIR_*).

Forward projections must be bit-identical, including multi-frame volumes with a mask.
Backprojections are within the scatter tolerance (relative L2 <= 1e-6). OSEM images are
within 1e-4 relative L2. Header files are byte-identical.
"""
import os
import subprocess

import numpy as np
import pytest

from fir_b200 import capi, interfile, workloads
from fir_b200.geometry import VolSpec

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "fir_b200", "bin")
FIR = os.path.join(ROOT, "oracle", "_ref")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run(bindir, exe, *args, cwd, extra_env=None):
    path = os.path.join(bindir, exe)
    if not os.access(path, os.X_OK):
        pytest.skip(f"{path} not built")
    env = dict(os.environ, OMP_NUM_THREADS="1", **(extra_env or {}))
    p = subprocess.run([path, *args], capture_output=True, text=True, cwd=cwd, env=env, timeout=600)
    assert p.returncode == 0, f"{path}: {p.stdout[-2000:]}{p.stderr[-2000:]}"
    return p


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    w = workloads.small()
    interfile.write_scanner(str(d / "scanner.scan"), w.scanner)
    x = workloads.activity(w)
    interfile.write_vol(str(d / "image"), w.vol, x)
    two = VolSpec(w.vol.size, w.vol.voxel, w.vol.offset, n_frames=2)
    interfile.write_vol(str(d / "image2"), two, np.concatenate([x, 2 * x + 0.5]))
    mask = (np.random.default_rng(1).random(x.shape) > 0.2).astype(np.float32)
    interfile.write_vol(str(d / "mask"), w.vol, mask)
    interfile.write_vol_header(str(d / "template.h33"), w.vol)
    interfile.write_proj_header(str(d / "template.hs"), w.proj)
    interfile.write_vol(str(d / "hu"), w.vol, workloads.hounsfield(w))
    return d, w, x


def fwd_params(d, name, vol, frames=None, mask=None):
    lines = ["!FORWARD PROJECTION PARAMETERS :=", f"input volume file := {vol}", "scanner file := scanner.scan",
             "output projection header := template.hs", f"output projection file name := {name}"]
    if frames:
        lines.append("frames to project := {" + ", ".join(str(f) for f in frames) + "}")
    if mask:
        lines.append(f"mask volume file := {mask}")
    lines.append("!END OF FORWARD PROJECTION PARAMETERS :=")
    p = d / f"{name}.par"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


def test_forward_projection_bit_identical_to_fir(files):
    d, w, x = files
    outs = {}
    for tag, bindir in (("ours", OURS), ("fir", FIR), ("dropin", DROPIN)):
        run(bindir, "FIR_ForwardProj", fwd_params(d, f"fwd_{tag}", "image.h33"), cwd=d)
        outs[tag] = (np.fromfile(d / f"fwd_{tag}.s", np.float32), (d / f"fwd_{tag}.hs").read_text())
    np.testing.assert_array_equal(outs["ours"][0], outs["fir"][0])
    np.testing.assert_array_equal(outs["dropin"][0], outs["fir"][0])
    assert outs["ours"][1] == outs["fir"][1].replace("fwd_fir", "fwd_ours")


def test_multiframe_masked_forward_bit_identical_to_fir(files):
    d, w, x = files
    for tag, bindir in (("ours", OURS), ("fir", FIR)):
        run(bindir, "FIR_ForwardProj", fwd_params(d, f"mf_{tag}", "image2.h33", frames=[1, 0], mask="mask.h33"), cwd=d)
    for f in (0, 1):
        a = np.fromfile(d / f"mf_ours_frame_{f}.s", np.float32)
        b = np.fromfile(d / f"mf_fir_frame_{f}.s", np.float32)
        np.testing.assert_array_equal(a, b)


def test_backprojection_matches_fir(files):
    d, w, x = files
    run(FIR, "FIR_ForwardProj", fwd_params(d, "bp_in", "image.h33"), cwd=d)
    for tag, bindir in (("ours", OURS), ("fir", FIR), ("dropin", DROPIN)):
        run(bindir, "FIR_BackProj", "bp_in.hs", "scanner.scan", "template.h33", f"bp_{tag}", cwd=d)
    ref = np.fromfile(d / "bp_fir.i33", np.float32)
    for tag in ("ours", "dropin"):
        got = np.fromfile(d / f"bp_{tag}.i33", np.float32)
        assert rel_l2(got, ref) <= 1e-6
        assert (d / f"bp_{tag}.h33").read_text() == (d / "bp_fir.h33").read_text().replace("bp_fir", f"bp_{tag}")


def osem_params(d, tag):
    p = d / f"osem_{tag}.par"
    p.write_text("\n".join([
        "!OSEM PARAMETERS :=",
        "input projection file := counts.hs",
        "scanner file := scanner.scan",
        "output volume header := template.h33",
        f"output volume file name := rec_{tag}",
        "number of iterations := 2",
        "number of subsets := 4",
        "save interval := 3",
        "convolution interval := 1",
        "convolution FHWM XYZ in mm := {4, 4, 4}",
        # with the extension, so that the flags "0 0" find the files again
        f"sensitivity map volume := sens_{tag}.h33",
        "attenuation volume in HU := hu.h33",
        f"attenuation correction factors := acf_{tag}.hs",
        "!END OF OSEM PARAMETERS :=",
    ]) + "\n")
    return str(p)


def test_osem_with_attenuation_matches_fir(files):
    d, w, x = files
    run(FIR, "FIR_ForwardProj", fwd_params(d, "truth", "image.h33"), cwd=d)
    truth = np.fromfile(d / "truth.s", np.float32)
    counts = workloads.poisson_counts(truth, w.counts, 11)
    interfile.write_proj(str(d / "counts"), w.proj, counts)
    for tag, bindir in (("ours", OURS), ("fir", FIR), ("dropin", DROPIN)):
        run(bindir, "FIR_OSEM", osem_params(d, tag), cwd=d)
    ref = np.fromfile(d / "rec_fir.i33", np.float32)
    for tag in ("ours", "dropin"):
        assert rel_l2(np.fromfile(d / f"rec_{tag}.i33", np.float32), ref) <= 1e-4
        assert rel_l2(np.fromfile(d / f"sens_{tag}.i33", np.float32), np.fromfile(d / "sens_fir.i33", np.float32)) <= 1e-6
        acf = np.fromfile(d / f"acf_{tag}.s", np.float32)
        acf_ref = np.fromfile(d / "acf_fir.s", np.float32)
        assert np.max(np.abs(acf.view(np.int32).astype(np.int64) - acf_ref.view(np.int32))) <= 1
        for k in (3, 6):
            inter = d / f"rec_{tag}_subiter_{k}.i33"
            assert inter.exists()
            assert rel_l2(np.fromfile(inter, np.float32),
                          np.fromfile(d / f"rec_fir_subiter_{k}.i33", np.float32)) <= 1e-4
    # flags 0 0: sensitivity and attenuation factors are read from the files
    first = np.fromfile(d / "rec_ours.i33", np.float32)
    run(OURS, "FIR_OSEM", osem_params(d, "ours"), "0", "0", cwd=d)
    assert rel_l2(np.fromfile(d / "rec_ours.i33", np.float32), first) <= 1e-6


def test_timing_json_line(files):
    """FIR_TIMING_JSON=1 makes our executables print one JSON timing line on
    stderr; without it they print none."""
    import json

    d, w, x = files
    p = run(OURS, "FIR_ForwardProj", fwd_params(d, "t_json", "image.h33"), cwd=d, extra_env={"FIR_TIMING_JSON": "1"})
    lines = [ln for ln in p.stderr.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stderr
    rec = json.loads(lines[0])
    assert rec["program"] == "FIR_ForwardProj"
    assert rec["projector_launches"] >= 1 and rec["projector_ms"] > 0 and rec["kernel_launches"] >= 1
    q = run(OURS, "FIR_ForwardProj", fwd_params(d, "t_nojson", "image.h33"), cwd=d)
    assert not [ln for ln in q.stderr.splitlines() if ln.startswith("{")]
