"""Seeded synthetic volumes for the registration workloads.

No public dataset is needed or used: these generators stand in for the
fMRI/T1 data the reference is run on, with the shapes, value ranges and
motion statistics of the benchmark workloads.  Volumes are float32 arrays of
shape (D, H, W) (x fastest in memory), series are (T, D, H, W).

Transform convention (matches the registration parameters): a volume is
*moved* by T(x) = c + A (x - c) + t, i.e. moved(x) = base(T(x)); the
registration of `moved` back onto `base` recovers the parameters of
T^-1: translation -A^-1 t and matrix A^-1 - I, about the centre c.
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage


def _rotation(ax: float, ay: float, az: float) -> np.ndarray:
    cx, sx = np.cos(ax), np.sin(ax)
    cy, sy = np.cos(ay), np.sin(ay)
    cz, sz = np.cos(az), np.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def base_volume(shape=(33, 64, 64), seed: int = 0, n_ellipsoids: int = 5) -> np.ndarray:
    """Smoothed white noise (sigma 2 voxels, rescaled to unit variance) plus
    `n_ellipsoids` solid ellipsoids of intensity U(200, 1000), centres
    uniform in the inner 60 % of each axis, semi-axes U(3, 12) voxels and
    random orientation."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D, H, W = shape
    noise = rng.standard_normal(shape)
    noise = ndimage.gaussian_filter(noise, 2.0, mode="constant")
    noise /= max(noise.std(), 1e-12)
    vol = noise
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    pts = np.stack([x, y, z], -1).astype(np.float64)
    for _ in range(n_ellipsoids):
        inten = rng.uniform(200.0, 1000.0)
        c = np.array([rng.uniform(0.2 * W, 0.8 * W), rng.uniform(0.2 * H, 0.8 * H),
                      rng.uniform(0.2 * D, 0.8 * D)])
        semi = rng.uniform(3.0, 12.0, 3)
        R = _rotation(*rng.uniform(0, 2 * np.pi, 3))
        local = (pts - c) @ R
        inside = ((local / semi) ** 2).sum(-1) <= 1.0
        vol = vol + inten * inside
    return vol.astype(np.float32)


def transform_volume(vol: np.ndarray, A: np.ndarray, t: np.ndarray) -> np.ndarray:
    """moved(x) = vol(c + A (x - c) + t), trilinear, clamped at the edges.
    Coordinates are (x, y, z) voxel indices."""
    D, H, W = vol.shape
    c = np.array([(W - 1) / 2.0, (H - 1) / 2.0, (D - 1) / 2.0])
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    p = np.stack([x, y, z], -1).astype(np.float64) - c
    q = p @ A.T + c + t
    coords = np.stack([q[..., 2], q[..., 1], q[..., 0]])
    out = ndimage.map_coordinates(vol.astype(np.float64), coords, order=1, mode="nearest")
    return out.astype(np.float32)


def true_params(A: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Registration parameters that undo T(x) = c + A(x - c) + t."""
    Ai = np.linalg.inv(A)
    tt = -Ai @ t
    P = Ai - np.eye(3)
    return np.concatenate([tt, P.reshape(-1)]).astype(np.float64)


def rms_displacement_error(p_est, p_true, shape) -> float:
    """RMS over all voxels of the distance between the sample points of two
    parameter vectors (voxels)."""
    D, H, W = shape
    c = np.array([(W - 1) / 2.0, (H - 1) / 2.0, (D - 1) / 2.0])
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    p = np.stack([x, y, z], -1).reshape(-1, 3).astype(np.float64) - c
    pe = np.asarray(p_est, np.float64)
    pt = np.asarray(p_true, np.float64)
    de = p @ pe[3:].reshape(3, 3).T + pe[:3]
    dt = p @ pt[3:].reshape(3, 3).T + pt[:3]
    return float(np.sqrt(((de - dt) ** 2).sum(-1).mean()))


def affine_pair(shape=(33, 64, 64), base_seed: int = 0, motion_seed: int = 1):
    """A base volume and a copy moved by a seeded affine: rotations
    U(-5, 5) degrees, translations U(-3, 3) voxels, scales U(0.97, 1.03),
    about the volume centre.  Returns (base, moved, true registration
    parameters)."""
    base = base_volume(shape, base_seed)
    rng = np.random.Generator(np.random.PCG64(motion_seed))
    ang = np.deg2rad(rng.uniform(-5.0, 5.0, 3))
    t = rng.uniform(-3.0, 3.0, 3)
    s = rng.uniform(0.97, 1.03, 3)
    A = _rotation(*ang) @ np.diag(s)
    return base, transform_volume(base, A, t), true_params(A, t)


def motion_series(T: int = 200, shape=(33, 64, 64), base_seed: int = 0, snr: float = 50.0,
                  max_translation: float = 2.0, max_rotation_deg: float = 2.0, noise: bool = True,
                  base: np.ndarray = None):
    """fMRI-like series: volume t is the base volume under a rigid motion
    drawn from seed 100 + t (translations U(+-2) voxels, rotations U(+-2)
    degrees) plus Rician noise at the given SNR (noise std = mean
    foreground intensity / snr; magnitude of a complex signal with
    independent Gaussian noise in both channels).  Returns (series (T,D,H,W),
    true parameters (T,12) of each volume's own motion).  `base` replaces
    the generated base volume (its shape is then the series' shape)."""
    if base is None:
        base = base_volume(shape, base_seed)
    base = np.asarray(base, np.float32)
    shape = base.shape
    fg = base[base > 100.0]
    s = (fg.mean() if fg.size else np.abs(base).mean()) / snr
    vols = np.empty((T,) + tuple(shape), np.float32)
    truth = np.empty((T, 12))
    for t in range(T):
        rng = np.random.Generator(np.random.PCG64(100 + t))
        tr = rng.uniform(-max_translation, max_translation, 3)
        ang = np.deg2rad(rng.uniform(-max_rotation_deg, max_rotation_deg, 3))
        A = _rotation(*ang)
        v = transform_volume(base, A, tr).astype(np.float64)
        if noise:
            n1 = rng.standard_normal(v.shape) * s
            n2 = rng.standard_normal(v.shape) * s
            v = np.sqrt((v + n1) ** 2 + n2 ** 2)
        vols[t] = v.astype(np.float32)
        truth[t] = true_params(A, tr)
    return vols, truth


def head_phantom(shape, seed: int = 0, scale=None) -> np.ndarray:
    """T1-like head: three nested ellipsoidal tissue classes at intensities
    300 / 600 / 900 (outer, middle, inner), a few inner ellipsoidal
    structures, a smooth multiplicative bias field (second-order polynomial,
    within +-20 %) and Gaussian noise of sigma 15.  `scale` (3 floats, voxels
    per unit) sets the head size; by default it fills ~80 % of the grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    D, H, W = shape
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    c = np.array([(W - 1) / 2.0, (H - 1) / 2.0, (D - 1) / 2.0])
    r = np.array([0.40 * W, 0.42 * H, 0.40 * D]) if scale is None else np.asarray(scale, np.float64)
    px, py, pz = (x - c[0]) / r[0], (y - c[1]) / r[1], (z - c[2]) / r[2]
    rho = np.sqrt(px * px + py * py + pz * pz)
    vol = np.zeros(shape)
    vol[rho <= 1.0] = 300.0
    vol[rho <= 0.85] = 600.0
    vol[rho <= 0.6] = 900.0
    for _ in range(6):
        cc = rng.uniform(-0.4, 0.4, 3)
        ax = rng.uniform(0.08, 0.2, 3)
        inside = ((px - cc[0]) / ax[0]) ** 2 + ((py - cc[1]) / ax[1]) ** 2 + ((pz - cc[2]) / ax[2]) ** 2 <= 1
        vol[inside & (rho <= 0.85)] = rng.choice([300.0, 600.0])
    coef = rng.uniform(-1, 1, 9)
    bias = (coef[0] * px + coef[1] * py + coef[2] * pz + coef[3] * px * py + coef[4] * py * pz +
            coef[5] * px * pz + coef[6] * px * px + coef[7] * py * py + coef[8] * pz * pz)
    bias = 1.0 + 0.2 * bias / max(np.abs(bias).max(), 1e-12)
    vol = vol * bias + rng.standard_normal(shape) * 15.0
    return vol.astype(np.float32)


def smooth_field(shape, seed: int = 200, max_mm: float = 6.0, sigma: float = 8.0) -> np.ndarray:
    """Smooth displacement field (3, D, H, W) in voxels (1 mm voxels):
    Gaussian-smoothed white noise scaled so the largest displacement
    magnitude is max_mm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    f = np.stack([ndimage.gaussian_filter(rng.standard_normal(shape), sigma, mode="nearest")
                  for _ in range(3)])
    mag = np.sqrt((f * f).sum(0)).max()
    return (f * (max_mm / max(mag, 1e-12))).astype(np.float32)


def warp_with_field(vol: np.ndarray, field: np.ndarray) -> np.ndarray:
    """vol sampled at x + field(x) (trilinear, clamped)."""
    D, H, W = vol.shape
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    coords = np.stack([z + field[2], y + field[1], x + field[0]])
    return ndimage.map_coordinates(vol.astype(np.float64), coords, order=1, mode="nearest").astype(np.float32)


def t1_template_pair(subject_shape=(170, 256, 256), template_shape=(182, 218, 182), seed: int = 0):
    """A subject T1-like head warped by a smooth field (seed 200, max 6 mm)
    and a template built the same way (different seed, no warp), both 1 mm.
    Shapes are (D, H, W).  Returns (subject, template, field)."""
    tpl = head_phantom(template_shape, seed=seed + 1)
    sub = head_phantom(subject_shape, seed=seed,
                       scale=np.array([0.40 * template_shape[2], 0.42 * template_shape[1],
                                       0.40 * template_shape[0]]))
    fld = smooth_field(subject_shape, seed=200 + seed, max_mm=6.0, sigma=max(2.0, min(subject_shape) / 20))
    return warp_with_field(sub, fld), tpl, fld


def relative_params(p_ref, p_t) -> np.ndarray:
    """Parameters that map volume t onto the reference volume when both are
    moved copies of one base: compose T_ref^-1 ... expressed as the
    registration parameters of t relative to ref (both given as the
    registration parameters that undo their own motion)."""
    def mat(p):
        M = np.eye(4)
        M[:3, :3] += np.asarray(p[3:], np.float64).reshape(3, 3)
        M[:3, 3] = p[:3]
        return M
    # aligned_t(x) = vol_t(G_t x) = base(T_t G_t x); base(y) = vol_ref(G_ref^-1 y)
    # registration of vol_t onto vol_ref: vol_t(G x) = vol_ref(x)
    #   vol_ref(x) = base(T_ref x) = vol_t(T_t^-1 T_ref x) = vol_t(G_t G_ref^-1 x)
    M = mat(p_t) @ np.linalg.inv(mat(p_ref))
    out = np.zeros(12)
    out[:3] = M[:3, 3]
    out[3:] = (M[:3, :3] - np.eye(3)).reshape(-1)
    return out


def first_level_dataset(T: int = 20, epi_shape=(33, 64, 64), epi_voxel=(3.0, 3.0, 3.5), t1_shape=(170, 256, 256),
                        t1_voxel=(1.0, 1.0, 1.0), mni_shape=(182, 218, 182), mni_voxel=(1.0, 1.0, 1.0),
                        seed: int = 0):
    """Inputs of the first-level preprocessing: one head drawn three times.
    The template is head_phantom(mni_shape, seed + 1); the T1 and the EPI
    base are head_phantom(seed) with the template head's size in mm at
    their own voxel sizes, so a T1 and an EPI of the same head overlap the
    template after resampling; the EPI series is that base under rigid
    motion (motion_series, translations up to 1 voxel, rotations up to 1
    degree) with Rician noise at SNR 50.  Shapes are (D, H, W), voxel sizes
    (x, y, z) in mm.  Returns (fmri (T, D, H, W), t1, mni, true motion
    (T, 12))."""
    mni = head_phantom(mni_shape, seed=seed + 1)
    radii_mm = np.array([0.40 * mni_shape[2] * mni_voxel[0], 0.42 * mni_shape[1] * mni_voxel[1],
                         0.40 * mni_shape[0] * mni_voxel[2]])
    t1 = head_phantom(t1_shape, seed=seed, scale=radii_mm / np.asarray(t1_voxel, np.float64))
    epi = head_phantom(epi_shape, seed=seed, scale=radii_mm / np.asarray(epi_voxel, np.float64))
    fmri, truth = motion_series(T, base=epi, max_translation=1.0, max_rotation_deg=1.0)
    return fmri, t1, mni, truth
