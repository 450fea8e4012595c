"""The OSEM sub-iteration entry point that allocates nothing.

Reconstruction services that reserve their whole GPU memory budget at
start-up, and hosts whose GPU memory belongs to their own pool allocator,
cannot let the library allocate device memory while they run.  For them
fir_osem_subiteration_noalloc takes its scratch from one static device array
and needs only device pointers.  These tests call it through the C ABI and
check, on calls in a row, that it gives the image fir_osem_subiteration gives
(relative L2 within 1e-5, the tolerance the sub-iteration tests use: the
backprojection sums in atomic order), that the shared accumulator starts from
zero on every call, and that oversized volumes and host memory are rejected.
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


def noalloc(torch, w, xy, z, y, img, sens_frame, prm, subset, subiter, bias=None):
    st = torch.cuda.current_stream().cuda_stream
    return capi.lib().fir_osem_subiteration_noalloc(
        C.byref(capi.proj_desc(w.proj)), C.c_void_p(xy.data_ptr()), C.c_void_p(z.data_ptr()),
        C.c_void_p(y.data_ptr()), C.c_void_p(bias.data_ptr()) if bias is not None else None,
        C.byref(capi.vol_desc(w.vol, 1)), C.c_void_p(img.data_ptr()), C.c_void_p(sens_frame.data_ptr()),
        C.byref(capi.osem_desc(prm)), subset, subiter, capi.FIR_GEOMETRY_REFERENCE, C.c_void_p(st))


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
