"""Differentiable registration: gradients of the filter-response SSD with
respect to the 12 affine parameters and to a displacement field, from the
adjoint kernels through torch.autograd, against central finite differences
of the FP64 oracle with a step of 1e-3 voxel (translations and field
values 1e-3; an affine matrix entry the step that moves no voxel by more
than 1e-3 voxel).  Bar: relative error <= 1e-3,
|g_gpu - g_fd| <= 1e-3 * max|g_fd| over the checked components.

Evaluated away from the grid (sub-voxel parameters / field) so that the
trilinear interpolant is differentiable at every sample point."""
import numpy as np
import pytest
import torch

from broccoli_b200 import autograd as AG
from broccoli_b200 import synthetic as S

pytestmark = pytest.mark.gpu
H_FD = 1e-3
SIGMA = 2.0
SHAPE = (20, 26, 24)


def _pair():
    sub, tpl, _ = S.t1_template_pair(SHAPE, SHAPE, seed=3)
    return sub.astype(np.float32), tpl.astype(np.float32)


def _fd_steps(shape):
    """Central-difference steps of the 12 parameters that move no voxel by
    more than 1e-3 voxel: 1e-3 for the translations, 1e-3 / (half extent of
    the coordinate it multiplies) for a matrix entry (column 0 multiplies
    x - (W-1)/2, column 1 y, column 2 z)."""
    D, H, W = shape
    half = [(W - 1) / 2.0, (H - 1) / 2.0, (D - 1) / 2.0]
    return np.array([H_FD] * 3 + [H_FD / half[(i - 3) % 3] for i in range(3, 12)])


def _params():
    p = np.zeros(12, np.float64)
    p[:3] = [0.31, -0.27, 0.43]
    p[3:] = np.array([0.011, -0.007, 0.004, 0.006, -0.013, 0.002, -0.005, 0.008, 0.009])
    return p


def test_filter_adjoint_is_the_transpose(ctx, lin_filters):
    """<F x, y> == <x, F^T y> for random x, y."""
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.standard_normal((2,) + SHAPE).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((2, 3) + SHAPE + (2,)).astype(np.float32)).cuda()
    xr = x.clone().requires_grad_(True)
    fx = AG.filter3d(xr, lin_filters)
    lhs = (fx.double() * y.double()).sum()
    lhs.backward()
    rhs = (x.double() * xr.grad.double()).sum()
    assert abs(float(lhs) - float(rhs)) <= 1e-4 * abs(float(lhs))


def test_affine_gradient_vs_fp64_finite_differences(orc, lin_filters):
    mov, ref = _pair()
    dev = torch.device("cuda")
    q_ref = AG.reference_responses(torch.from_numpy(ref).to(dev), lin_filters, SIGMA)
    p = torch.tensor(_params(), dtype=torch.float32, device=dev, requires_grad=True)
    loss = AG.registration_objective(torch.from_numpy(mov).to(dev), q_ref, lin_filters, SIGMA, params=p)
    loss.backward()
    g = p.grad.cpu().numpy().astype(np.float64)
    p0 = _params()
    steps = _fd_steps(mov.shape)
    fd = np.zeros(12)
    for i in range(12):
        e = np.zeros(12)
        e[i] = steps[i]
        fd[i] = (orc.registration_objective(mov, ref, lin_filters, SIGMA, params=p0 + e) -
                 orc.registration_objective(mov, ref, lin_filters, SIGMA, params=p0 - e)) / (2 * steps[i])
    assert np.abs(g - fd).max() <= 1e-3 * np.abs(fd).max(), (g, fd)


def test_field_gradient_vs_fp64_finite_differences(orc, lin_filters):
    mov, ref = _pair()
    dev = torch.device("cuda")
    rng = np.random.default_rng(1)
    field = (rng.uniform(-0.45, 0.45, (3,) + SHAPE) + 0.05).astype(np.float64)
    q_ref = AG.reference_responses(torch.from_numpy(ref).to(dev), lin_filters, SIGMA)
    f = torch.tensor(field, dtype=torch.float32, device=dev, requires_grad=True)
    loss = AG.registration_objective(torch.from_numpy(mov).to(dev), q_ref, lin_filters, SIGMA, field=f)
    loss.backward()
    g = f.grad.cpu().numpy().astype(np.float64)
    # a seeded random subset of interior voxels, all three components
    D, H, W = SHAPE
    picks = [(c, rng.integers(4, D - 4), rng.integers(4, H - 4), rng.integers(4, W - 4))
             for c in range(3) for _ in range(3)]
    fd, gg = [], []
    for c, z, y, x in picks:
        fp = field.copy()
        fm = field.copy()
        fp[c, z, y, x] += H_FD
        fm[c, z, y, x] -= H_FD
        fd.append((orc.registration_objective(mov, ref, lin_filters, SIGMA, field=fp) -
                   orc.registration_objective(mov, ref, lin_filters, SIGMA, field=fm)) / (2 * H_FD))
        gg.append(g[c, z, y, x])
    fd = np.array(fd)
    gg = np.array(gg)
    assert np.abs(gg - fd).max() <= 1e-3 * np.abs(fd).max(), (gg, fd)


def test_moving_volume_gradient_vs_finite_differences(orc, lin_filters):
    """Gradient with respect to the moving volume (smoothing adjoint +
    scatter adjoint of the warp), checked at a few voxels."""
    mov, ref = _pair()
    dev = torch.device("cuda")
    q_ref = AG.reference_responses(torch.from_numpy(ref).to(dev), lin_filters, SIGMA)
    m = torch.from_numpy(mov).to(dev).requires_grad_(True)
    p = torch.tensor(_params(), dtype=torch.float32, device=dev)
    loss = AG.registration_objective(m, q_ref, lin_filters, SIGMA, params=p)
    loss.backward()
    g = m.grad.cpu().numpy().astype(np.float64)
    mv = mov.astype(np.float64)
    fd, gg = [], []
    h = 1e-2
    for z, y, x in [(10, 13, 12), (8, 9, 15), (12, 17, 7)]:
        a = mv.copy()
        b = mv.copy()
        a[z, y, x] += h
        b[z, y, x] -= h
        fd.append((orc.registration_objective(a, ref, lin_filters, SIGMA, params=_params()) -
                   orc.registration_objective(b, ref, lin_filters, SIGMA, params=_params())) / (2 * h))
        gg.append(g[z, y, x])
    fd = np.array(fd)
    assert np.abs(np.array(gg) - fd).max() <= 1e-3 * np.abs(fd).max()


def test_gradients_at_full_config_size(orc, lin_filters):
    """The differentiable-registration workload's own size: a 128x128x96 pair
    made as the T1-like template pair, smoothing sigma 2.  All 12 affine
    gradients and the field gradient at six seeded interior voxels (all
    three components) against FP64 central differences of the oracle (steps
    of 1e-3 voxel); bar 1e-3 of the largest finite difference, as above."""
    shape = (96, 128, 128)
    sub, tpl, _ = S.t1_template_pair(shape, shape, seed=3)
    mov, ref = sub.astype(np.float32), tpl.astype(np.float32)
    dev = torch.device("cuda")
    q_ref = AG.reference_responses(torch.from_numpy(ref).to(dev), lin_filters, SIGMA)
    p = torch.tensor(_params(), dtype=torch.float32, device=dev, requires_grad=True)
    AG.registration_objective(torch.from_numpy(mov).to(dev), q_ref, lin_filters, SIGMA, params=p).backward()
    g = p.grad.cpu().numpy().astype(np.float64)
    p0 = _params()
    steps = _fd_steps(mov.shape)
    fd = np.zeros(12)
    for i in range(12):
        e = np.zeros(12)
        e[i] = steps[i]
        fd[i] = (orc.registration_objective(mov, ref, lin_filters, SIGMA, params=p0 + e) -
                 orc.registration_objective(mov, ref, lin_filters, SIGMA, params=p0 - e)) / (2 * steps[i])
    assert np.abs(g - fd).max() <= 1e-3 * np.abs(fd).max(), (g, fd)

    rng = np.random.default_rng(7)
    field = (rng.uniform(-0.45, 0.45, (3,) + shape) + 0.05).astype(np.float64)
    f = torch.tensor(field, dtype=torch.float32, device=dev, requires_grad=True)
    AG.registration_objective(torch.from_numpy(mov).to(dev), q_ref, lin_filters, SIGMA, field=f).backward()
    gf = f.grad.cpu().numpy().astype(np.float64)
    D, H, W = shape
    picks = [(c, int(rng.integers(8, D - 8)), int(rng.integers(8, H - 8)), int(rng.integers(8, W - 8)))
             for c in range(3) for _ in range(2)]
    fdf, gg = [], []
    for c, z, y, x in picks:
        fp, fm = field.copy(), field.copy()
        fp[c, z, y, x] += H_FD
        fm[c, z, y, x] -= H_FD
        fdf.append((orc.registration_objective(mov, ref, lin_filters, SIGMA, field=fp) -
                    orc.registration_objective(mov, ref, lin_filters, SIGMA, field=fm)) / (2 * H_FD))
        gg.append(gf[c, z, y, x])
    fdf, gg = np.array(fdf), np.array(gg)
    assert np.abs(gg - fdf).max() <= 1e-3 * np.abs(fdf).max(), (gg, fdf)
