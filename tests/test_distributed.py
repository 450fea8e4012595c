"""Multi-process OSEM (fir_b200.distributed) on CPU with gloo, world size 2.

Each rank backprojects its share of every subset with a CPU backend built
on the oracle.  The all-reduce sums the shares, and every rank applies the
same update.

The result must match the single-process oracle OSEM within 1e-5 relative
L2; only the order of the float sum of the two shares differs.  Both ranks
must hold bit-identical images.

A rank that fails before an exchange must make the other rank fail with an
error within the process-group timeout instead of hanging.
"""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fir_b200 import workloads
from fir_b200.geometry import OSEMParams

EPS = 1e-5


class OracleBackend:
    """The five operations ShardedOSEM needs, on CPU tensors, by the oracle."""

    def __init__(self, w):
        from oracle.bridge import Restated

        self.R = Restated()
        self.w = w

    def ratio_backprojection(self, proj, sino, vol, img, bp, n_subsets, subset, bias=None, n_shards=1, shard=0):
        w = self.w
        line = self.R.forward(w.scanner, proj, vol, img.numpy())
        if bias is not None:
            line = (line + bias.numpy()).astype(np.float32)
        y = sino.numpy()
        ok = line.astype(np.float64) > EPS
        ratio = np.zeros_like(line)
        ratio[ok] = y[ok] / line[ok]
        # bins of the other views backproject a ratio of exactly 0
        views = view_of_bins(self.R, proj)
        k = views // n_subsets
        ratio[~((views % n_subsets == subset) & (k % n_shards == shard))] = 0.0
        frames = self.R.backward(w.scanner, proj, vol, ratio, 1)
        bp.copy_(torch.from_numpy(frames.copy()))

    def em_update(self, vol, img, bp, sens):
        a, b = self.R.em_update(img.numpy(), bp.numpy(), sens.numpy())
        img.copy_(torch.from_numpy(a))
        bp.copy_(torch.from_numpy(b))

    def convolve(self, vol, img, fwhm, cut):
        img.copy_(torch.from_numpy(self.R.convolve(vol, img.numpy(), fwhm, cut)))

    def cut_circle(self, vol, img, cut):
        img.copy_(torch.from_numpy(self.R.cut_circle(vol, img.numpy(), cut)))


def view_of_bins(R, proj):
    """View index of every bin, FIR's file order (segments of [view][axial][tang])."""
    f = R.proj(proj)
    parts = []
    for k in range(proj.n_segments):
        parts.append(np.repeat(np.arange(f.n_views), f.n_axial[k] * f.n_tang_coords))
    return np.concatenate(parts)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def problem():
    w = workloads.tiny()
    prm = OSEMParams(n_iterations=2, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=55.0)
    return w, prm


def _rank_main(rank, world, port, outdir, fail_rank, exchange="all_reduce"):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from fir_b200.distributed import ShardedOSEM
    from oracle.bridge import Restated

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        w, prm = problem()
        R = Restated()
        x = workloads.activity(w)
        y = workloads.poisson_counts(R.forward(w.scanner, w.proj, w.vol, x), w.counts, 4)
        sens = R.sensitivity(w.scanner, w.proj, w.vol, prm.n_subsets).reshape(prm.n_subsets, *w.vol.shape_zyx)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the first exchange")
        img = torch.ones(w.vol.shape_zyx, dtype=torch.float32)
        ShardedOSEM(OracleBackend(w), w.proj, w.vol, prm, exchange=exchange).run(torch.from_numpy(y), img,
                                                                                 torch.from_numpy(sens))
        np.save(os.path.join(outdir, f"img{rank}.npy"), img.numpy())
    except Exception as e:  # noqa: BLE001
        with open(os.path.join(outdir, f"err{rank}.txt"), "w") as f:
            f.write(repr(e))
        raise
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _launch(world, fail_rank=-1, deadline=240, exchange="all_reduce"):
    outdir = tempfile.mkdtemp(prefix="firdist_")
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, outdir, fail_rank, exchange))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(deadline)
    hung = [p.pid for p in procs if p.is_alive()]
    for p in procs:
        if p.is_alive():
            p.kill()
    return outdir, [p.exitcode for p in procs], hung


@pytest.mark.parametrize("world,exchange", [(2, "all_reduce"), (3, "all_reduce"), (2, "reduce_scatter"),
                                            (3, "reduce_scatter")])
def test_sharded_osem_matches_single_process_oracle(restated, world, exchange):
    """World 3 splits each subset's 8 views 3 + 3 + 2 and the 8 slices of the
    image into slabs of 3, 3 and 2."""
    outdir, codes, hung = _launch(world, exchange=exchange)
    errs = [open(os.path.join(outdir, f"err{r}.txt")).read() for r in range(world)
            if os.path.exists(os.path.join(outdir, f"err{r}.txt"))]
    assert not hung and codes == [0] * world, errs or codes
    a = np.load(os.path.join(outdir, "img0.npy"))
    for r in range(1, world):
        np.testing.assert_array_equal(a, np.load(os.path.join(outdir, f"img{r}.npy")))
    w, prm = problem()
    x = workloads.activity(w)
    y = workloads.poisson_counts(restated.forward(w.scanner, w.proj, w.vol, x), w.counts, 4)
    sens = restated.sensitivity(w.scanner, w.proj, w.vol, prm.n_subsets)
    want = restated.osem(w.scanner, w.proj, w.vol, y, np.ones_like(x), sens, prm)
    assert np.linalg.norm(a - want) <= 1e-5 * np.linalg.norm(want)


def test_failed_rank_is_reported_not_hung():
    outdir, codes, hung = _launch(2, fail_rank=1, deadline=120)
    assert not hung
    assert codes[1] != 0
    # the surviving rank leaves its exchange with an error instead of waiting forever
    assert codes[0] != 0
    assert os.path.exists(os.path.join(outdir, "err0.txt"))


def test_shard_mapping():
    from fir_b200.distributed import Shard

    # rank r takes the subset's k-th view for k % world == r: the shares
    # partition the subset's views v % n == s for any world size, evenly or not
    n, n_views = 4, 32
    for world in (1, 2, 3, 5, 8, 9):
        for s in range(n):
            shares = [Shard(r, world).views(s, n, n_views) for r in range(world)]
            flat = sorted(v for sh in shares for v in sh)
            assert flat == [v for v in range(n_views) if v % n == s]
            sizes = [len(sh) for sh in shares]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    # slabs cover the slices once, the last ones possibly short or empty
    for nz, world in ((8, 3), (64, 8), (5, 8)):
        covered = []
        for r in range(world):
            z0, z1, per = Shard(r, world).slab(nz)
            assert z1 - z0 <= per and per * world >= nz
            covered += list(range(z0, z1))
        assert covered == list(range(nz))
