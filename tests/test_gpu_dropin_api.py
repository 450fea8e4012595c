"""FIR's C++ API over the GPU: a program written against FIR's headers
(ProjData::getBinCoordinates, ProjData::rebinWeight, the bin accessors) is
compiled against the drop-in headers, linked with libfir / libfir_cuda, and
run.  Its results must equal the C restatement of FIR (itself pinned to
compiled FIR)."""
import os
import subprocess

import numpy as np
import pytest

from fir_b200 import interfile
from fir_b200.geometry import ProjSpec

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <ProjData.h>
#include <cstdio>
#include <fstream>

// argv: header, pairs file (n x 4 ints), output prefix
int main(int argc, char** argv)
{
  ProjData proj(argv[1], ProjData::ConstructionMode::INITIALIZE, 1.0f);
  std::ifstream in(argv[2]);
  std::FILE* out = std::fopen((std::string(argv[3]) + "_bins.txt").c_str(), "w");
  int r1, c1, r2, c2;
  while (in >> r1 >> c1 >> r2 >> c2)
  {
    int seg = 0, view = 0, axial = 0, tang = 0;
    const bool ok = proj.getBinCoordinates(r1, c1, r2, c2, &seg, &view, &axial, &tang);
    std::fprintf(out, "%d %d %d %d %d\n", ok ? 1 : 0, ok ? seg : 0, ok ? view : 0, ok ? axial : 0, ok ? tang : 0);
  }
  std::fclose(out);
  // weight an all-ones sinogram, then read every bin back through the accessors
  proj.rebinWeight();
  const auto& g = proj.getGeometry();
  std::FILE* w = std::fopen((std::string(argv[3]) + "_weights.bin").c_str(), "wb");
  for (int seg = -g.segOffset; seg <= g.segOffset; ++seg)
    for (int view = 0; view < g.nViews; ++view)
      for (int ax = 0; ax < g.getNAxialCoords(seg); ++ax)
        for (int t = -g.tangCoordOffset; t < -g.tangCoordOffset + proj.getHeader().nTangCoords; ++t)
        {
          const float v = proj.getBin(seg, view, ax, t);
          std::fwrite(&v, sizeof(float), 1, w);
        }
  std::fclose(w);
  return 0;
}
"""


def test_cpp_bin_coordinates_and_rebin_weight(tmp_path, restated):
    src = tmp_path / "prog.cc"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    lib = os.path.join(ROOT, "fir_b200", "lib")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "fir_b200", "csrc", "host", "include"),
           "-I", os.path.join(ROOT, "include"), str(src), "-L", lib, "-lfir", "-lfir_cuda",
           f"-Wl,-rpath,{lib}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    p = ProjSpec(8, 128, 5, 61, 3)
    interfile.write_proj_header(str(tmp_path / "p.hs"), p)
    rng = np.random.default_rng(12)
    pairs = np.stack([rng.integers(0, 8, 3000), rng.integers(0, 128, 3000), rng.integers(0, 8, 3000),
                      rng.integers(0, 128, 3000)], axis=1)
    np.savetxt(tmp_path / "pairs.txt", pairs, fmt="%d")
    r = subprocess.run([str(exe), str(tmp_path / "p.hs"), str(tmp_path / "pairs.txt"), str(tmp_path / "out")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.loadtxt(tmp_path / "out_bins.txt", dtype=np.int32).reshape(-1, 5)
    np.testing.assert_array_equal(got, restated.bin_coordinates(p, pairs))
    n = restated.proj(p).n_bins
    weights = np.fromfile(tmp_path / "out_weights.bin", np.float32)
    np.testing.assert_array_equal(weights, restated.rebin_weight(p, np.ones(n, np.float32)))
