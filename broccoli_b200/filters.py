"""Quadrature filter banks for phase-based registration.

The reference ships optimised 7x7x7 complex filters as raw float32 files
(``filters/filter{k}_{real,imag}_{linear,nonlinear}_registration.bin``, 343
values each, x fastest) plus projection tensors and filter directions for
the nonlinear stage.  :func:`load_filter_dir` reads a directory laid out that
way.  :func:`lognormal_quadrature_filters` designs filters of our own
(lognormal radial function, cos^2 directional function, truncated to 7^3),
used for workloads that ask for a given centre frequency and bandwidth
rather than the shipped coefficients.

Filter bank arrays have shape (nfilt, 2, 7, 7, 7): filter, re/im, z, y, x.
"""
from __future__ import annotations

import os

import numpy as np

FILTER_SIZE = 7


def lognormal_quadrature_filters(directions, u0: float = np.pi / 3, bandwidth_octaves: float = 2.0,
                                 size: int = FILTER_SIZE, grid: int = 64) -> np.ndarray:
    """Spatial quadrature filters with frequency response
    R(rho) * D(u . n) where R(rho) = exp(-4 ln^2(rho/u0) / (B^2 ln 2)) and
    D(c) = c^2 for c > 0, 0 otherwise.  The response is sampled on a grid^3
    DFT grid, transformed to the spatial domain and truncated to size^3 about
    the origin; the DC leakage of the truncation is removed from the real
    part so that the filter stays blind to the local mean."""
    dirs = np.asarray(directions, dtype=np.float64)
    k = np.fft.fftfreq(grid) * 2.0 * np.pi
    uz, uy, ux = np.meshgrid(k, k, k, indexing="ij")
    rho = np.sqrt(ux * ux + uy * uy + uz * uz)
    with np.errstate(divide="ignore", invalid="ignore"):
        radial = np.exp(-4.0 * np.log(rho / u0) ** 2 / (bandwidth_octaves ** 2 * np.log(2.0)))
    radial[rho == 0] = 0.0
    h = size // 2
    out = np.zeros((len(dirs), 2, size, size, size), np.float64)
    for i, n in enumerate(dirs):
        n = n / np.linalg.norm(n)
        with np.errstate(invalid="ignore", divide="ignore"):
            c = (ux * n[0] + uy * n[1] + uz * n[2]) / rho
        c[rho == 0] = 0.0
        F = radial * np.where(c > 0, c * c, 0.0)
        f = np.fft.ifftn(F)
        f = np.fft.fftshift(f)
        m = grid // 2
        crop = f[m - h:m + h + 1, m - h:m + h + 1, m - h:m + h + 1]
        crop = crop / np.abs(crop).max()
        re = crop.real - crop.real.mean()
        out[i, 0] = re
        out[i, 1] = crop.imag
    return out.astype(np.float32)


def linear_registration_filters(u0: float = np.pi / 3, bandwidth_octaves: float = 2.0) -> np.ndarray:
    """Three filters along x, y and z (the layout the affine stage expects:
    filter k senses displacement along axis k)."""
    return lognormal_quadrature_filters(np.eye(3), u0, bandwidth_octaves)


def _read_bin(path: str, count: int) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float32)
    if a.size != count:
        raise ValueError(f"{path}: expected {count} float32 values, found {a.size}")
    return a


def load_filter_dir(path: str):
    """Read the reference's filter directory layout.

    Returns a dict with ``linear`` (3,2,7,7,7), ``nonlinear`` (6,2,7,7,7),
    ``projection_tensors`` (6,6: m11 m12 m13 m22 m23 m33) and
    ``directions`` (3,6: x, y, z components of the six filter directions)."""
    n = FILTER_SIZE ** 3
    out = {}
    lin = np.zeros((3, 2, 7, 7, 7), np.float32)
    for k in range(3):
        lin[k, 0] = _read_bin(os.path.join(path, f"filter{k + 1}_real_linear_registration.bin"), n).reshape(7, 7, 7)
        lin[k, 1] = _read_bin(os.path.join(path, f"filter{k + 1}_imag_linear_registration.bin"), n).reshape(7, 7, 7)
    out["linear"] = lin
    nl_path = os.path.join(path, "filter1_real_nonlinear_registration.bin")
    if os.path.exists(nl_path):
        nl = np.zeros((6, 2, 7, 7, 7), np.float32)
        for k in range(6):
            nl[k, 0] = _read_bin(os.path.join(path, f"filter{k + 1}_real_nonlinear_registration.bin"), n).reshape(7, 7, 7)
            nl[k, 1] = _read_bin(os.path.join(path, f"filter{k + 1}_imag_nonlinear_registration.bin"), n).reshape(7, 7, 7)
        out["nonlinear"] = nl
        out["projection_tensors"] = np.stack(
            [_read_bin(os.path.join(path, f"projection_tensor{k + 1}.bin"), 6) for k in range(6)])
        out["directions"] = np.stack(
            [_read_bin(os.path.join(path, f"filter_directions_{a}.bin"), 6) for a in "xyz"])
    return out
