"""4D transforms on the GPU (brc_transform_volumes_linear / _nonlinear,
brc_center_volumes, brc_change_resolution_and_size_batch,
brc_combine_displacement_field) against the reference's kernels (golden
vectors, tests/golden/transforms.npz) and the oracle.

The transform kernels form coordinates and trilinear weights in the
reference's operation order with every operation rounded, so the results
are expected bit for bit: with NEAREST a different rounding would pick
another voxel."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from broccoli_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return dict(np.load(os.path.join(GOLDEN, "transforms.npz")))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("interp,tag", [(L.INTERP_NEAREST, "nearest"), (L.INTERP_LINEAR, "linear")])
def test_transforms_match_golden(ctx, g, interp, tag):
    v = cuda(g["vols"])
    a = ctx.transform_volumes_linear(v, g["p12"], interp).cpu().numpy()
    assert np.array_equal(a, g["affine_" + tag])
    f = ctx.transform_volumes_nonlinear(v, *(cuda(x) for x in g["field"]), interpolation=interp).cpu().numpy()
    assert np.array_equal(f, g["field_" + tag])
    c, p = ctx.center_volumes(v, interp)
    assert np.array_equal(p, g["center_p12_" + tag])
    assert np.array_equal(c.cpu().numpy(), g["center_" + tag])
    r = ctx.change_resolution_and_size_batch(v, g["vin"], tuple(g["shape2"]), g["vnew"], int(g["zcut"]), interp)
    assert np.array_equal(r.cpu().numpy(), g["resize_" + tag])


def test_combined_field_matches_golden(ctx, g):
    f = [cuda(x) for x in g["field"]]
    ctx.combine_displacement_field(*f, g["p12"])
    assert np.array_equal(np.stack([x.cpu().numpy() for x in f]), g["combined_field"])


@pytest.mark.parametrize("shape,T", [((7, 9, 13), 1), ((20, 17, 11), 4), ((3, 40, 5), 2)])
@pytest.mark.parametrize("interp", [L.INTERP_NEAREST, L.INTERP_LINEAR])
def test_transforms_match_oracle_odd_shapes(ctx, orc, shape, T, interp):
    rng = np.random.default_rng(sum(shape) + T + interp)
    v = (rng.standard_normal((T,) + shape) * 30 + 80).astype(np.float32)
    p = (rng.standard_normal(12) * np.r_[1.5, 1.5, 1.5, [0.03] * 9]).astype(np.float32)
    fld = (rng.standard_normal((3,) + shape) * 2).astype(np.float32)
    assert np.array_equal(ctx.transform_volumes_linear(cuda(v), p, interp).cpu().numpy(),
                          orc.transform_affine(v, p, interp))
    assert np.array_equal(ctx.transform_volumes_nonlinear(cuda(v), *(cuda(x) for x in fld),
                                                          interpolation=interp).cpu().numpy(),
                          orc.transform_field(v, *fld, interp=interp))
    r = ctx.change_resolution_and_size_batch(cuda(v), (1.0, 1.5, 2.0), (9, 12, 8), (1.25, 1.25, 1.5), 0, interp)
    assert np.array_equal(r.cpu().numpy(),
                          orc.change_resolution_and_size_interp(v, (1.0, 1.5, 2.0), (9, 12, 8), (1.25, 1.25, 1.5),
                                                                0, interp))


def test_cubic_and_bad_arguments_are_refused(ctx, g):
    v = cuda(g["vols"])
    with pytest.raises(L.BrcError) as e:
        ctx.transform_volumes_linear(v, g["p12"], L.INTERP_CUBIC)
    assert e.value.status == L.BRC_ERR_UNSUPPORTED
    with pytest.raises(L.BrcError) as e:
        ctx.center_volumes(v, 7)
    assert e.value.status == L.BRC_ERR_INVALID
    with pytest.raises(L.BrcError) as e:
        ctx.change_resolution_and_size_batch(v, (1, 1, 0), (4, 4, 4), (1, 1, 1))
    assert e.value.status == L.BRC_ERR_INVALID


def test_python_class_transform_wrappers(g):
    """BROCCOLI_LIB.TransformVolumesLinear/NonLinearWrapper and
    CenterVolumesWrapper through the Python class (setter interface)."""
    from broccoli_b200 import broccoli_lib as B
    v = g["vols"]
    T, D, H, W = v.shape
    lib = B.BROCCOLI_LIB(0, 0)
    lib.SetT1Width(W); lib.SetT1Height(H); lib.SetT1Depth(D); lib.SetT1Timepoints(T)
    for f, x in zip((lib.SetT1VoxelSizeX, lib.SetT1VoxelSizeY, lib.SetT1VoxelSizeZ), g["vin"]):
        f(x)
    D2, H2, W2 = (int(x) for x in g["shape2"])
    lib.SetMNIWidth(W2); lib.SetMNIHeight(H2); lib.SetMNIDepth(D2)
    for f, x in zip((lib.SetMNIVoxelSizeX, lib.SetMNIVoxelSizeY, lib.SetMNIVoxelSizeZ), g["vnew"]):
        f(x)
    lib.SetMMT1ZCUT(int(g["zcut"]))
    lib.SetInputT1Volume(np.ascontiguousarray(v))
    lib.SetInterpolationMode(B.NEAREST)
    params = np.ascontiguousarray(g["p12"])
    out = np.zeros((T, D2, H2, W2), np.float32)
    lib.SetOutputT1MNIRegistrationParameters(params)
    lib.SetOutputInterpolatedT1Volume(out)
    lib.TransformVolumesLinearWrapper()
    expect = np.stack([g["resize_nearest"][t] for t in range(T)])
    import oracle
    assert np.array_equal(out, oracle.transform_affine(expect, params, 0))
    centred = np.zeros_like(v)
    lib.SetOutputInterpolatedT1Volume(centred)
    lib.CenterVolumesWrapper()
    assert np.array_equal(centred, g["center_nearest"])
    assert np.array_equal(lib.center_parameters, g["center_p12_nearest"])
    with pytest.raises(ValueError):
        lib.SetInterpolationMode(B.CUBIC)
