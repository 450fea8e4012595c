"""The OSEM sub-iteration entry point that allocates nothing.

Reconstruction services that reserve their whole GPU memory budget at
start-up, and hosts whose GPU memory belongs to their own pool allocator,
cannot let the library allocate device memory while they run.  For them
fir_osem_subiteration_noalloc takes its scratch from one static device array
and needs only device pointers.  These tests call it through the C ABI and
check, on calls in a row, that it gives the image fir_osem_subiteration gives
(relative L2 within 1e-5, the tolerance the sub-iteration tests use: the
backprojection sums in atomic order) in both geometry modes and with the
filter skipped, that the shared accumulator starts from zero on every call,
that calls after the first leave the device's free memory unchanged, and that
oversized volumes and host memory are rejected.
"""
import ctypes as C

import numpy as np
import pytest

from fir_b200 import capi, workloads
from fir_b200.geometry import OSEMParams, VolSpec

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def noalloc(torch, w, xy, z, y, img, sens_frame, prm, subset, subiter, bias=None,
            geometry=capi.FIR_GEOMETRY_REFERENCE, vol=None):
    st = torch.cuda.current_stream().cuda_stream
    return capi.lib().fir_osem_subiteration_noalloc(
        C.byref(capi.proj_desc(w.proj)), C.c_void_p(xy.data_ptr()), C.c_void_p(z.data_ptr()),
        C.c_void_p(y.data_ptr()), C.c_void_p(bias.data_ptr()) if bias is not None else None,
        C.byref(capi.vol_desc(vol or w.vol, 1)), C.c_void_p(img.data_ptr()), C.c_void_p(sens_frame.data_ptr()),
        C.byref(capi.osem_desc(prm)), subset, subiter, geometry, C.c_void_p(st))


@pytest.fixture(scope="module")
def setup():
    import torch

    assert torch.cuda.is_available()
    w = workloads.small()
    ctx = capi.Context(w.scanner)
    x = torch.from_numpy(workloads.activity(w)).cuda()
    ax = torch.empty(w.n_lors, device="cuda")
    ctx.forward(w.vol, x, w.proj, ax)
    gen = torch.Generator(device="cuda").manual_seed(3)
    y = torch.poisson(ax * (w.counts / float(ax.sum())), generator=gen)
    sens = torch.empty((4,) + w.vol.shape_zyx, device="cuda")
    ctx.sensitivity(w.proj, w.vol, sens, 4)
    xy_h, z_h = capi.scanner_tables(w.scanner)
    xy = torch.from_numpy(np.ascontiguousarray(xy_h)).cuda()
    z = torch.from_numpy(z_h).cuda()
    prm = OSEMParams(n_iterations=1, n_subsets=4, convolution_interval=1, fwhm_xyz=[4.0, 4.0, 4.0],
                     cut_radius=110.0)
    yield torch, w, ctx, y, sens, xy, z, prm
    ctx.close()


def test_noalloc_matches_context_entry_point_on_calls_in_a_row(setup):
    torch, w, ctx, y, sens, xy, z, prm = setup
    start = torch.ones(w.vol.shape_zyx, device="cuda")
    ref = start.clone()
    got = start.clone()
    bias = torch.full((w.n_lors,), 0.01, device="cuda")
    for k, subset in enumerate((0, 1, 2)):
        ctx.osem_subiteration(w.proj, y, w.vol, ref, sens[subset].contiguous(), prm, subset, k + 1, bias=bias)
        rc = noalloc(torch, w, xy, z, y, got, sens[subset].contiguous(), prm, subset, k + 1, bias=bias)
        assert rc == 0, capi.lib().fir_last_error().decode()
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= TOL
    # the same first sub-iteration again: the shared accumulator starts at zero
    again = start.clone()
    assert noalloc(torch, w, xy, z, y, again, sens[0].contiguous(), prm, 0, 1, bias=bias) == 0
    first = start.clone()
    ctx.osem_subiteration(w.proj, y, w.vol, first, sens[0].contiguous(), prm, 0, 1, bias=bias)
    torch.cuda.synchronize()
    assert rel_l2(again.cpu().numpy(), first.cpu().numpy()) <= TOL


@pytest.mark.parametrize("geometry,interval", [(capi.FIR_GEOMETRY_EXACT, 1), (capi.FIR_GEOMETRY_REFERENCE, 2)])
def test_noalloc_exact_geometry_and_skipped_filter(setup, geometry, interval):
    """A volume of 3.5 mm voxels in FIR_GEOMETRY_EXACT (real extents), and a
    filter interval of 2, whose odd sub-iterations skip the filter: both
    against fir_osem_subiteration of a context in the same mode."""
    torch, w, ctx, y, sens, xy, z, prm = setup
    vol = VolSpec.centred((64, 64, 16), (3.5, 3.5, 3.5)) if geometry == capi.FIR_GEOMETRY_EXACT else w.vol
    p2 = OSEMParams(n_iterations=1, n_subsets=4, convolution_interval=interval, fwhm_xyz=[4.0, 4.0, 4.0],
                    cut_radius=110.0)
    with capi.Context(w.scanner) as c2:
        c2.set_option(capi.FIR_OPT_GEOMETRY, geometry)
        s2 = torch.empty((4,) + vol.shape_zyx, device="cuda")
        c2.sensitivity(w.proj, vol, s2, 4)
        ref = torch.ones(vol.shape_zyx, device="cuda")
        got = ref.clone()
        for k, subset in enumerate((0, 1, 2)):
            c2.osem_subiteration(w.proj, y, vol, ref, s2[subset].contiguous(), p2, subset, k + 1)
            rc = noalloc(torch, w, xy, z, y, got, s2[subset].contiguous(), p2, subset, k + 1, geometry=geometry,
                         vol=vol)
            assert rc == 0, capi.lib().fir_last_error().decode()
            torch.cuda.synchronize()
            assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_noalloc_allocates_nothing(setup):
    """After a first call, further calls change neither the device's free
    memory nor torch's allocator statistics."""
    torch, w, ctx, y, sens, xy, z, prm = setup
    img = torch.ones(w.vol.shape_zyx, device="cuda")
    frames = [sens[k].contiguous() for k in range(4)]
    assert noalloc(torch, w, xy, z, y, img, frames[0], prm, 0, 1) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = torch.cuda.memory_stats()
    for k in range(1, 4):
        assert noalloc(torch, w, xy, z, y, img, frames[k], prm, k, k + 1) == 0, capi.lib().fir_last_error().decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = torch.cuda.memory_stats()
    assert free1 == free0
    for key in ("allocation.all.allocated", "reserved_bytes.all.current", "allocated_bytes.all.current"):
        assert stats1.get(key, 0) == stats0.get(key, 0), key


def test_noalloc_rejects_oversized_volumes_and_host_memory(setup):
    torch, w, ctx, y, sens, xy, z, prm = setup
    big = VolSpec.centred((128, 128, 65), (4.0, 4.0, 4.0))  # 1064960 voxels > 1 << 20
    img = torch.ones(big.shape_zyx, device="cuda")
    frame = torch.ones(big.shape_zyx, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = capi.lib().fir_osem_subiteration_noalloc(
        C.byref(capi.proj_desc(w.proj)), C.c_void_p(xy.data_ptr()), C.c_void_p(z.data_ptr()),
        C.c_void_p(y.data_ptr()), None, C.byref(capi.vol_desc(big, 1)), C.c_void_p(img.data_ptr()),
        C.c_void_p(frame.data_ptr()), C.byref(capi.osem_desc(prm)), 0, 1, capi.FIR_GEOMETRY_REFERENCE,
        C.c_void_p(st))
    assert rc == 1  # FIR_ERR_INVALID_ARGUMENT
    assert "no-allocation limit of 1048576 voxels" in capi.lib().fir_last_error().decode()
    host_img = np.ones(w.vol.shape_zyx, np.float32)
    rc = capi.lib().fir_osem_subiteration_noalloc(
        C.byref(capi.proj_desc(w.proj)), C.c_void_p(xy.data_ptr()), C.c_void_p(z.data_ptr()),
        C.c_void_p(y.data_ptr()), None, C.byref(capi.vol_desc(w.vol, 1)), C.c_void_p(host_img.ctypes.data),
        C.c_void_p(sens[0].data_ptr()), C.byref(capi.osem_desc(prm)), 0, 1, capi.FIR_GEOMETRY_REFERENCE,
        C.c_void_p(st))
    assert rc == 1 and "must be device memory" in capi.lib().fir_last_error().decode()
