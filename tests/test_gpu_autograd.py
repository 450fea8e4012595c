"""The differentiable projector (fir_b200.autograd) and the multi-frame
projectors under it (fir_forward_frames / fir_backward_frames).

* float32 frames equal FIR's per-frame projection bit for bit, and the
  per-frame backprojection up to the order of the float atomics (1e-6
  relative L2);
* adjoint dot-product test <Ax, y> = <x, A^T y> on random non-negative x, y:
  1e-5 relative in float32, 1e-12 in float64;
* the gradient of the penalized Poisson NLL agrees with central finite
  differences (h = 1e-3, 64 random voxels) to 1e-3 relative, in float64;
* the NLL gradient equals FIR's own BackProj of the ratio sinogram
  a * (1 - y / ybar) to 1e-5 relative L2;
* L-BFGS lowers the penalized NLL.

The finite-difference and FIR-BackProj checks run on the small workload and
again at the differentiable-projector workload's scale (clinical scanner,
3.28e7 LORs, one 128x128x48 phantom).
"""
import numpy as np
import pytest
import torch

from fir_b200 import autograd as fa
from fir_b200 import workloads

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def small():
    w = workloads.small()
    op = fa.SiddonProjector(w.scanner, w.proj, w.vol)
    yield w, op
    op.close()


def rand_images(w, n, seed, dtype=torch.float32):
    g = torch.Generator(device=DEV).manual_seed(seed)
    return torch.rand((n,) + tuple(w.vol.shape_zyx), generator=g, device=DEV, dtype=dtype)


def test_forward_frames_bit_identical_to_forward(small):
    w, op = small
    for n in (3, 9):
        x = rand_images(w, n, 1)
        y = op.project(x)
        for f in range(n):
            want = torch.empty(op.n_bins, device=DEV)
            op.ctx.forward(w.vol, x[f].contiguous(), w.proj, want)
            assert torch.equal(y[f], want), f


def test_backward_frames_matches_backward(small):
    w, op = small
    g = torch.Generator(device=DEV).manual_seed(2)
    y = torch.rand(5, op.n_bins, generator=g, device=DEV)
    x = op.backproject(y)
    for f in range(5):
        want = torch.empty(w.vol.shape_zyx, device=DEV)
        op.ctx.backward(w.proj, y[f].contiguous(), w.vol, want, 1)
        assert float((x[f] - want).norm() / want.norm()) <= 1e-6


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 1e-5), (torch.float64, 1e-12)])
def test_adjoint_dot_product(small, dtype, tol):
    w, op = small
    x = rand_images(w, 2, 3, dtype)
    g = torch.Generator(device=DEV).manual_seed(4)
    y = torch.rand(2, op.n_bins, generator=g, device=DEV, dtype=dtype)
    lhs = float((op.project(x).double() * y.double()).sum())
    rhs = float((x.double() * op.backproject(y).double()).sum())
    assert abs(lhs - rhs) <= tol * abs(lhs)


def _data(w, op, dtype):
    """Attenuation factors and Poisson data of the workload's phantom."""
    from fir_b200 import capi

    mu = torch.from_numpy(workloads.hounsfield(w)).to(DEV)
    op.ctx.hu_to_mu(w.vol, mu)
    acf = torch.empty(op.n_bins, device=DEV)
    op.ctx.forward_exp(w.vol, mu, w.proj, acf)
    atten = (1.0 / acf).to(dtype)
    x_true = torch.from_numpy(workloads.activity(w)).to(DEV)
    ybar = op.project(x_true) * (1.0 / acf)
    ybar *= w.counts / float(ybar.sum())
    y = torch.poisson(ybar, generator=torch.Generator(device=DEV).manual_seed(w.seed)).to(dtype)
    scale = w.counts / float((op.project(x_true) * (1.0 / acf)).sum())
    return atten * scale, y, x_true.to(dtype)


def test_gradient_matches_finite_differences(small):
    w, op = small
    atten, y, x_true = _data(w, op, torch.float64)
    x = (0.5 + 0.5 * rand_images(w, 1, 5, torch.float64)[0]).requires_grad_(True)
    beta = 0.01
    loss = fa.penalized_nll(x, y, op, beta, atten)
    loss.backward()
    grad = x.grad.detach()
    rng = np.random.default_rng(6)
    nz, ny, nx = w.vol.shape_zyx
    h = 1e-3
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            j = (int(rng.integers(nz)), int(rng.integers(ny)), int(rng.integers(nx)))
            xp = x.detach().clone()
            xp[j] += h
            xm = x.detach().clone()
            xm[j] -= h
            fd = (float(fa.penalized_nll(xp, y, op, beta, atten)) - float(fa.penalized_nll(xm, y, op, beta, atten))) \
                / (2 * h)
            g = float(grad[j])
            worst = max(worst, abs(fd - g) / max(abs(g), 1e-3))
    assert worst <= 1e-3, worst


def test_nll_gradient_equals_fir_backprojection_of_ratio(small, reference):
    w, op = small
    atten, y, _ = _data(w, op, torch.float32)
    x = (0.5 + rand_images(w, 1, 7)[0]).requires_grad_(True)
    ybar = fa.expected_counts(x, op, atten)
    fa.poisson_nll(ybar, y).backward()
    with torch.no_grad():
        ratio = ((1.0 - y / ybar) * atten).cpu().numpy()
    want = reference.backward(w.scanner, w.proj, w.vol, ratio, 1).reshape(w.vol.shape_zyx)
    got = x.grad.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)


def test_lbfgs_lowers_the_objective(small):
    w, op = small
    atten, y, x_true = _data(w, op, torch.float32)
    x, stats = fa.reconstruct_lbfgs(op, y, 0.01, atten, steps=10)
    assert stats["evaluations"] >= 10
    assert stats["losses"][-1] < stats["losses"][0]
    assert torch.isfinite(x).all() and float(x.min()) >= 0.0
    c = np.corrcoef(x.cpu().numpy().ravel(), x_true.cpu().numpy().ravel())[0, 1]
    assert c > 0.3, c  # 10 steps from a uniform start: partly converged


# ---- the same checks at the differentiable-projector workload's scale: the
# clinical scanner (32 rings x 512 crystals, 125 tangential bins, 3.28e7
# LORs) and one 128x128x48 phantom at 3 mm with water attenuation

@pytest.fixture(scope="module")
def clinical_frame():
    w = workloads.autograd_batch(1)[0]
    op = fa.SiddonProjector(w.scanner, w.proj, w.vol)
    yield w, op
    op.close()


def loss_difference(xp, xm, y, op, beta, atten):
    """penalized_nll(xp) - penalized_nll(xm), summed bin by bin: at 3.28e7
    bins the loss is ~1e9 and the rounding of each total alone (~1e-6) would
    swamp a central difference with h = 1e-3, while the per-bin differences
    vanish exactly outside the LORs through the perturbed voxel."""
    def terms(x):
        yb = fa.expected_counts(x, op, atten)
        return yb - torch.xlogy(y, yb)

    return float((terms(xp) - terms(xm)).sum()) + float(fa.quadratic_penalty(xp, beta) - fa.quadratic_penalty(xm, beta))


def test_gradient_matches_finite_differences_at_scale(clinical_frame):
    """Central differences, h = 1e-3, on 64 random voxels of the field of
    view, float64: 1e-3 relative."""
    w, op = clinical_frame
    atten, y, x_true = _data(w, op, torch.float64)
    x = (0.5 + 0.5 * rand_images(w, 1, 15, torch.float64)[0]).requires_grad_(True)
    beta = 0.01
    loss = fa.penalized_nll(x, y, op, beta, atten)
    loss.backward()
    grad = x.grad.detach()
    rng = np.random.default_rng(16)
    nz, ny, nx = w.vol.shape_zyx
    h = 1e-3
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            # within 45 voxels (135 mm) of the axis, inside the 150 mm field of view
            while True:
                j = (int(rng.integers(nz)), int(rng.integers(ny)), int(rng.integers(nx)))
                if (j[1] - ny / 2) ** 2 + (j[2] - nx / 2) ** 2 < 45 ** 2:
                    break
            xp = x.detach().clone()
            xp[j] += h
            xm = x.detach().clone()
            xm[j] -= h
            fd = loss_difference(xp, xm, y, op, beta, atten) / (2 * h)
            g = float(grad[j])
            worst = max(worst, abs(fd - g) / max(abs(g), 1e-3))
    assert worst <= 1e-3, worst


def test_nll_gradient_equals_fir_backprojection_at_scale(clinical_frame, reference):
    """The NLL gradient of the float32 path against FIR's own BackProj of the
    ratio sinogram (oracle/_ref, all host threads): 1e-5 relative L2."""
    import os

    w, op = clinical_frame
    atten, y, _ = _data(w, op, torch.float32)
    x = (0.5 + rand_images(w, 1, 17)[0]).requires_grad_(True)
    ybar = fa.expected_counts(x, op, atten)
    fa.poisson_nll(ybar, y).backward()
    with torch.no_grad():
        ratio = ((1.0 - y / ybar) * atten).cpu().numpy()
    reference.threads(os.cpu_count() or 1)
    want = reference.backward(w.scanner, w.proj, w.vol, ratio, 1).reshape(w.vol.shape_zyx)
    got = x.grad.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
