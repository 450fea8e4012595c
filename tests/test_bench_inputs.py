"""The benchmark's two arms run on the same inputs, and the reference arm runs
FIR's own code only.

bench.py's GPU arm makes its measured sinogram from this library's forward
projections, its reference arm from FIR's (oracle/_ref); both pass them through
workloads.measured_sinogram.  The forward projections are bit-identical, so
the sinograms are too.  On the CPU the restatement stands in for the GPU
projector (it is pinned bit for bit to FIR); the GPU test uses the GPU."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _inputs(project, w, nb, hu_to_mu):
    from fir_b200 import workloads

    mu = hu_to_mu(workloads.hounsfield(w))
    line_mu = project(mu)
    ax = project(workloads.activity(w))
    return workloads.measured_sinogram(w, ax, line_mu)


def test_measured_sinogram_identical_from_fir_and_restatement(reference, restated):
    from fir_b200 import workloads

    w = workloads.small()
    nb = reference.proj_geometry(w.proj)["n_bins"]
    y_ref = _inputs(lambda im: reference.forward(w.scanner, w.proj, w.vol, im, nb), w, nb,
                    lambda hu: reference.hu_to_mu(w.vol, hu))
    y_res = _inputs(lambda im: restated.forward(w.scanner, w.proj, w.vol, im), w, nb, restated.hu_to_mu)
    assert y_ref.shape == (nb,)
    assert np.array_equal(y_ref, y_res)
    # the data are counts times correction factors >= 1, with zeros where no count fell
    assert float(y_ref.min()) == 0.0 and 0.5e6 < float(y_ref.sum()) < 5e6


def test_reference_arm_loads_only_fir(reference):
    """bench.py --impl reference on the small workload: one JSON line with the
    GPU arm's config keys, and no library of fir_b200 mapped in the process."""
    probe = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'small', '--steps', '4']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('MAPPED', 'libfir_cuda' in maps, 'libfirref' in maps)\n"
    )
    p = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert set(d["config"]) == {"workload", "l2", "parallelism"}
    assert d["cpu_baseline"]["kind"] == "reference"
    assert "MAPPED False True" in p.stdout


@pytest.mark.gpu
def test_measured_sinogram_identical_on_gpu(reference):
    import torch

    from fir_b200 import capi, workloads

    w = workloads.small()
    nb = reference.proj_geometry(w.proj)["n_bins"]
    y_ref = _inputs(lambda im: reference.forward(w.scanner, w.proj, w.vol, im, nb), w, nb,
                    lambda hu: reference.hu_to_mu(w.vol, hu))
    with capi.Context(w.scanner) as ctx:
        def project(im):
            out = torch.empty(nb, device="cuda:0")
            ctx.forward(w.vol, torch.from_numpy(np.ascontiguousarray(im)).to("cuda:0"), w.proj, out)
            return out.cpu().numpy()

        def hu_to_mu(hu):
            t = torch.from_numpy(np.ascontiguousarray(hu)).to("cuda:0")
            ctx.hu_to_mu(w.vol, t)
            return t.cpu().numpy()

        y_gpu = _inputs(project, w, nb, hu_to_mu)
    assert np.array_equal(y_ref, y_gpu)
