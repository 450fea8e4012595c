"""The precision study that decides the traversal's arithmetic.

FP64 is kept in the Siddon traversal only if single precision changes the
voxel lists.  The oracle traverses sampled clinical LORs with FIR's double
arithmetic and with a float loop (after FIR's double set-up, and with a float
set-up too) and counts the LORs whose voxel lists differ.  They do, for a few
per cent of clinical LORs, with line integrals off by up to about 1 %, so the
GPU traversal replays FIR's double arithmetic (and its lists are bit-identical
to FIR's, tests/test_gpu_parity.py)."""
import numpy as np
import pytest

from fir_b200 import workloads


@pytest.mark.parametrize("precision", [1, 2])
def test_float_traversal_changes_voxel_lists(restated, precision):
    w = workloads.clinical()
    nb = restated.proj(w.proj).n_bins
    bins = np.sort(np.random.default_rng(0).choice(nb, 50000, replace=False)).astype(np.int64)
    r = restated.precision_study(w.scanner, w.proj, w.vol, workloads.activity(w), bins, precision)
    assert r["lors"] == 50000
    share = r["lists_differ"] / r["lors"]
    assert 0.005 < share < 0.1, r
    assert r["max_rel_line"] > 1e-3, r
