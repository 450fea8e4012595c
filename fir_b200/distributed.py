"""OSEM sharded over GPUs: one process per GPU, torch.distributed for plumbing.

FIR runs on one process.  Its sub-iteration has one exchange step: the
backprojection image is a sum over the subset's LORs.  Here the views of each
subset are split across ranks: rank r takes the subset's k-th view for every
k with k % world == r (subset s holds views v with v % n == s,
LORCache.cc:49-51), so the shares partition the subset for any number of
ranks; when world does not divide the subset's views, the first ranks hold
one view more.  Each sub-iteration then does:

1. every rank backprojects measured/estimated over its share
   (fir_ratio_backprojection_shard);
2. the exchange, one of:
   - ``"all_reduce"`` (default): one all-reduce (sum) of the backprojection
     image; every rank then applies the same gated EM update, filter and cut,
     so the images stay identical without further communication;
   - ``"reduce_scatter"``: a reduce-scatter of the backprojection into z
     slabs, the gated EM update of each rank's slab only, and an all-gather
     of the updated image; every rank then filters and cuts the whole image.
     It moves the same bytes as the all-reduce and does the EM update once
     instead of on every rank.  The filter runs after the all-gather because
     its z pass needs the neighbouring slabs.

The exchanges use NCCL over NVLink for CUDA tensors, and gloo in the CPU
tests.  An all-reduce moves nx*ny*nz floats per sub-iteration: 10 MB for the
clinical image, tens of microseconds on NVLink 5.

The compute backend is a :class:`fir_b200.capi.Context` in production.  Tests
inject a CPU backend with the same methods.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import torch
import torch.distributed as dist

from .geometry import OSEMParams, ProjSpec, VolSpec

EXCHANGES = ("all_reduce", "reduce_scatter")


@dataclass
class Shard:
    rank: int
    world: int

    def views(self, subset: int, n_subsets: int, n_views: int):
        """The views of `subset` (of `n_subsets`) that this rank backprojects."""
        return list(range(subset + n_subsets * self.rank, n_views, n_subsets * self.world))

    def slab(self, nz: int):
        """Slices [z0, z1) of this rank's slab, and the padded slab depth."""
        per = -(-nz // self.world)
        z0 = min(nz, self.rank * per)
        return z0, min(nz, z0 + per), per


def current_shard(group=None) -> Shard:
    if dist.is_available() and dist.is_initialized():
        return Shard(dist.get_rank(group), dist.get_world_size(group))
    return Shard(0, 1)


class ShardedOSEM:
    """reconAlgos::OSEM (reconAlgos.cc:63-201) with each subset's views split
    across the ranks of `group`.

    backend: object with ratio_backprojection (with n_shards / shard),
    em_update, convolve, cut_circle (the signatures of
    fir_b200.capi.Context).  exchange: one of EXCHANGES.
    """

    def __init__(self, backend, proj: ProjSpec, vol: VolSpec, params: OSEMParams, group=None,
                 exchange: str = "all_reduce"):
        if exchange not in EXCHANGES:
            raise ValueError(f"exchange must be one of {EXCHANGES}")
        self.backend = backend
        self.proj = proj
        self.vol = vol
        self.params = params
        self.group = group
        self.exchange = exchange
        self.shard = current_shard(group)
        nx, ny, nz = (int(v) for v in vol.size)
        self.nxy = nx * ny
        self.z0, self.z1, self.per = self.shard.slab(nz)
        self.slab_vol = VolSpec((nx, ny, self.z1 - self.z0), vol.voxel, vol.offset)
        self._padded = None

    def _exchange(self, img, bp, sens_frame):
        """Sum of the ranks' backprojections and the gated EM update; returns
        this rank's part of the backprojection divided by the sensitivity."""
        w = self.shard.world
        if w == 1 or self.exchange == "all_reduce":
            if w > 1:
                dist.all_reduce(bp, op=dist.ReduceOp.SUM, group=self.group)
            self.backend.em_update(self.vol, img, bp, sens_frame)
            return bp
        n = self.nxy * self.per
        if self._padded is None or self._padded.device != bp.device:
            self._padded = torch.zeros(w * n, dtype=bp.dtype, device=bp.device)
        full = self._padded
        full[: bp.numel()].copy_(bp.reshape(-1))
        part = torch.empty(n, dtype=bp.dtype, device=bp.device)
        dist.reduce_scatter_tensor(part, full, op=dist.ReduceOp.SUM, group=self.group)
        lo, hi = self.z0 * self.nxy, self.z1 * self.nxy
        flat = img.reshape(-1)
        if hi > lo:
            mine = flat[lo:hi].clone()
            bpm = part[: hi - lo].clone()
            self.backend.em_update(self.slab_vol, mine, bpm, sens_frame.reshape(-1)[lo:hi].clone())
            part[: hi - lo].copy_(bpm)
            piece = torch.zeros(n, dtype=img.dtype, device=img.device)
            piece[: hi - lo].copy_(mine)
        else:
            piece = torch.zeros(n, dtype=img.dtype, device=img.device)
        gathered = torch.empty(w * n, dtype=img.dtype, device=img.device)
        dist.all_gather_into_tensor(gathered, piece, group=self.group)
        flat.copy_(gathered[: flat.numel()])
        return part[: hi - lo]

    def subiteration(self, sino, img, sens_frame, subset: int, subiter: int, bias=None,
                     bp: Optional[torch.Tensor] = None) -> torch.Tensor:
        """One sub-iteration in place on img; returns the summed backprojection
        divided by the sensitivity (the whole image for the all-reduce, this
        rank's slab for the reduce-scatter), as fir_em_update leaves it."""
        p = self.params
        if bp is None:
            bp = torch.zeros_like(img)
        self.backend.ratio_backprojection(self.proj, sino, self.vol, img, bp, p.n_subsets, subset, bias=bias,
                                          n_shards=self.shard.world, shard=self.shard.rank)
        out = self._exchange(img, bp, sens_frame)
        conv = p.convolution_interval > 0 and all(f > 0 for f in p.fwhm_xyz)
        if conv and subiter % p.convolution_interval == 0:
            self.backend.convolve(self.vol, img, p.fwhm_xyz, p.cut_radius)
        if p.cut_radius > 0:
            self.backend.cut_circle(self.vol, img, p.cut_radius)
        return out

    def run(self, sino, img, sens, bias=None, save=None) -> None:
        """The full loop: initial cut, then n_iterations x n_subsets
        sub-iterations; sens holds n_subsets frames.  save(subiter, img) is
        called on rank 0 at the save interval."""
        p = self.params
        if p.cut_radius > 0:
            self.backend.cut_circle(self.vol, img, p.cut_radius)
        total = p.n_iterations * p.n_subsets
        bp = torch.zeros_like(img)
        for it in range(p.n_iterations):
            for s in range(p.n_subsets):
                k = it * p.n_subsets + s + 1
                bp.zero_()
                self.subiteration(sino, img, sens[s], s, k, bias=bias, bp=bp)
                if save is not None and p.save_interval > 0 and k % p.save_interval == 0 and k != total \
                        and self.shard.rank == 0:
                    save(k, img)
