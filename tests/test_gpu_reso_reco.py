"""FIR's OSEM_ResoReco (reconAlgos.cc:203-367) as FIR runs it, on the GPU.

Three forms are compared with FIR's own compiled function on the small
workload (2 iterations x 4 subsets, bias, cut radius, post-filter):
- the C ABI entry fir_osem_reso_reco, float atomics: image within 1e-4
  relative L2, filtered sensitivity bit-identical;
- the same entry in deterministic backprojection mode: image and sensitivity
  bit-identical to FIR run on one thread;
- FIR's C++ API (reconAlgos::OSEM_ResoReco of the drop-in layer) in a program
  compiled against the drop-in headers, reading and writing FIR's files.
The ABI test also counts the context's kernel launches: the loop runs on the
device.
"""
import os
import subprocess

import numpy as np
import pytest

from fir_b200 import capi, interfile, workloads
from fir_b200.geometry import OSEMParams

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PRM = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=2, fwhm_xyz=[4.0, 4.0, 4.0], cut_radius=110.0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case(reference, restated):
    w = workloads.small()
    x = workloads.activity(w)
    nb = reference.proj_geometry(w.proj)["n_bins"]
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 4)
    sens4 = restated.sensitivity(w.scanner, w.proj, w.vol, 4).reshape(4, -1)
    sens = np.concatenate([sens4, sens4.sum(axis=0, keepdims=True)]).reshape(-1, *x.shape[1:])  # 5 frames
    bias = np.full(nb, 0.02, np.float32)
    reference.threads(1)
    img_ref, sens_ref = reference.osem_reso_reco(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, PRM,
                                                 bias=bias)
    reference.threads(os.cpu_count() or 1)
    return w, x, y, sens, bias, img_ref, sens_ref


@pytest.mark.parametrize("mode", [capi.FIR_BACKPROJ_ATOMIC, capi.FIR_BACKPROJ_DETERMINISTIC])
def test_abi_reso_reco_matches_fir(case, mode):
    import torch

    w, x, y, sens, bias, img_ref, sens_ref = case
    with capi.Context(w.scanner) as ctx:
        ctx.set_option(capi.FIR_OPT_BACKPROJ_MODE, mode)
        img = torch.ones(w.vol.shape_zyx, device="cuda:0")
        dsens = torch.from_numpy(sens.copy()).to("cuda:0")
        launches0 = ctx.launch_count
        ctx.osem_reso_reco(w.proj, torch.from_numpy(y).to("cuda:0"), w.vol, img, dsens, PRM, n_sens_frames=5,
                           bias=torch.from_numpy(bias).to("cuda:0"))
        ctx.synchronize()
        launches = ctx.launch_count - launches0
        got, got_sens = img.cpu().numpy(), dsens.cpu().numpy()
    np.testing.assert_array_equal(got_sens.ravel(), sens_ref)
    if mode == capi.FIR_BACKPROJ_DETERMINISTIC:
        np.testing.assert_array_equal(got, img_ref)
    else:
        assert rel_l2(got, img_ref) <= 1e-4
    assert launches >= 8 * 3  # projector, filter and EM kernels of every sub-iteration


def test_abi_reso_reco_host_buffers(case):
    """Host (pageable) buffers are staged once: same result as device buffers."""
    w, x, y, sens, bias, img_ref, sens_ref = case
    with capi.Context(w.scanner) as ctx:
        img = np.ones(w.vol.shape_zyx, np.float32)
        s = sens.copy()
        ctx.osem_reso_reco(w.proj, y, w.vol, img, s, PRM, n_sens_frames=5, bias=bias)
    np.testing.assert_array_equal(s.ravel(), sens_ref)
    assert rel_l2(img, img_ref) <= 1e-4


PROGRAM = r"""
#include <ProjData.h>
#include <ScannerData.h>
#include <VolData.h>
#include <reconAlgos.h>
#include <optional>
#include <string>

// argv: scanner, sinogram header, bias header, sensitivity, initial image, output prefix
int main(int argc, char** argv)
{
  ScannerData scanner(argv[1]);
  ProjData proj(argv[2], ProjData::ConstructionMode::READ_DATA);
  std::optional<ProjData> bias;
  bias.emplace(argv[3], ProjData::ConstructionMode::READ_DATA);
  VolData sens(argv[4], VolData::ConstructionMode::READ_DATA);
  VolData vol(argv[5], VolData::ConstructionMode::READ_DATA);
  OSEMCoreParams params;
  params.nIterations = 2;
  params.nSubsets = 4;
  params.convolutionInterval = 2;
  params.cutRadius = 110.0f;
  params.fwhmXYZ = {4.0f, 4.0f, 4.0f};
  const std::string out(argv[6]);
  reconAlgos::OSEM_ResoReco(proj, scanner, vol, out, params, sens, bias);
  vol.write(out + "_image.h33");
  sens.write(out + "_sens.h33");
  return sens.getActiveFrame() == 3 ? 0 : 3;
}
"""


def test_cpp_reso_reco_dropin_matches_fir(case, tmp_path):
    w, x, y, sens, bias, img_ref, sens_ref = case
    src = tmp_path / "reso.cc"
    src.write_text(PROGRAM)
    exe = tmp_path / "reso"
    lib = os.path.join(ROOT, "fir_b200", "lib")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "fir_b200", "csrc", "host", "include"),
           "-I", os.path.join(ROOT, "include"), str(src), "-L", lib, "-lfir", "-lfir_cuda",
           f"-Wl,-rpath,{lib}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    d = tmp_path
    interfile.write_scanner(str(d / "s.scan"), w.scanner)
    interfile.write_proj(str(d / "y"), w.proj, y)
    interfile.write_proj(str(d / "bias"), w.proj, bias)
    interfile.write_vol(str(d / "sens"), w.vol.with_frames(5), sens)
    interfile.write_vol(str(d / "init"), w.vol, np.ones_like(x))
    r = subprocess.run([str(exe), str(d / "s.scan"), str(d / "y.hs"), str(d / "bias.hs"), str(d / "sens.h33"),
                        str(d / "init.h33"), str(d / "out")], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, FIR_TIMING_JSON="1"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    _, got = interfile.read_vol(str(d / "out_image.h33"))
    _, got_sens = interfile.read_vol(str(d / "out_sens.h33"))
    np.testing.assert_array_equal(got_sens.ravel(), sens_ref)
    assert rel_l2(got, img_ref) <= 1e-4


def test_abi_reso_reco_rejects_too_few_sensitivity_frames(case):
    """FIR's setActiveFrame(subset) fails with "Invalid frame" when the
    sensitivity volume has fewer frames than subsets."""
    w, x, y, sens, bias, img_ref, sens_ref = case
    with capi.Context(w.scanner) as ctx:
        img = np.ones(w.vol.shape_zyx, np.float32)
        with pytest.raises(capi.FirError, match="Invalid frame"):
            ctx.osem_reso_reco(w.proj, y, w.vol, img, sens.copy(), PRM, n_sens_frames=3)
