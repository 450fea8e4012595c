"""The multi-GPU share of a subset on one GPU: fir_ratio_backprojection_shard.

The shares of n_shards ranks partition a subset's views for any n_shards; the
sum of their backprojections must equal the subset's (fir_ratio_backprojection)
up to the order of the float additions (relative L2 <= 1e-6), also when
n_shards does not divide the subset's views, and a shard without views gives
zeros.  A ShardedOSEM of one rank must equal fir_osem."""
import numpy as np
import pytest

from fir_b200 import capi, workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n_shards", [2, 3, 5, 17])
def test_shards_sum_to_the_subset(n_shards):
    import torch

    w = workloads.small()  # 64 views, 4 subsets of 16 views
    with capi.Context(w.scanner) as ctx:
        nb = capi.proj_geometry(w.proj)["n_bins"]
        x = torch.from_numpy(workloads.activity(w)).cuda() + 0.05
        ax = torch.empty(nb, device="cuda")
        ctx.forward(w.vol, x, w.proj, ax)
        y = torch.poisson(ax * 3.0, generator=torch.Generator(device="cuda").manual_seed(2))
        img = torch.ones(w.vol.shape_zyx, device="cuda")
        whole = torch.empty_like(img)
        ctx.ratio_backprojection(w.proj, y, w.vol, img, whole, 4, 1)
        total = torch.zeros_like(img)
        part = torch.empty_like(img)
        empty = 0
        for r in range(n_shards):
            ctx.ratio_backprojection(w.proj, y, w.vol, img, part, 4, 1, n_shards=n_shards, shard=r)
            if float(part.abs().sum()) == 0.0:
                empty += 1
            total += part
        torch.cuda.synchronize()
        assert rel_l2(total.cpu().numpy(), whole.cpu().numpy()) <= 1e-6
        assert empty == max(0, n_shards - 16)


def test_sharded_osem_one_rank_is_fir_osem():
    import torch

    from fir_b200.distributed import ShardedOSEM

    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        ctx.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
        nb = capi.proj_geometry(w.proj)["n_bins"]
        x = torch.from_numpy(workloads.activity(w)).cuda()
        ax = torch.empty(nb, device="cuda")
        ctx.forward(w.vol, x, w.proj, ax)
        y = torch.poisson(ax * 3.0, generator=torch.Generator(device="cuda").manual_seed(2))
        sens = torch.empty((4,) + w.vol.shape_zyx, device="cuda")
        ctx.sensitivity(w.proj, w.vol, sens, 4)
        prm = w.osem
        a = torch.ones(w.vol.shape_zyx, device="cuda")
        ctx.osem(w.proj, y, w.vol, a, sens, prm)
        b = torch.ones(w.vol.shape_zyx, device="cuda")
        ShardedOSEM(ctx, w.proj, w.vol, prm).run(y, b, sens)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_shard_arguments_checked():
    import torch

    w = workloads.small()
    with capi.Context(w.scanner) as ctx:
        nb = capi.proj_geometry(w.proj)["n_bins"]
        y = torch.ones(nb, device="cuda")
        img = torch.ones(w.vol.shape_zyx, device="cuda")
        bp = torch.empty_like(img)
        for n_shards, shard in ((0, 0), (3, 3), (3, -1)):
            with pytest.raises(capi.FirError, match="shard"):
                ctx.ratio_backprojection(w.proj, y, w.vol, img, bp, 4, 1, n_shards=n_shards, shard=shard)
        with pytest.raises(capi.FirError):
            ctx.ratio_backprojection(w.proj, y, w.vol, img, bp, 5, 1, n_shards=2, shard=0)  # 5 does not divide 64 views
