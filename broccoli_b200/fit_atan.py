"""Coefficients of the arctangent polynomial used by the phase kernels.

atan(t) on t in [0, 1] is approximated as t * P(t^2), P of degree 8, with
the coefficients chosen to minimise the largest RELATIVE error (the phase
differences near convergence are small angles, so relative accuracy is what
the normal equations see).  The minimax fit is found by Lawson's iteration:
weighted least squares whose weights are multiplied by the current error at
every step, on a Chebyshev-spaced grid.  `python -m broccoli_b200.fit_atan`
prints the coefficients in the form csrc/common.cuh holds them and the
float32 error of that evaluation.
"""
import numpy as np

NTERMS = 9


def fit(nterms=NTERMS, iters=300, npts=20001):
    t = np.sort(np.cos(np.linspace(0.0, np.pi, npts)) * 0.5 + 0.5)
    t = t[t > 0]
    f = np.arctan(t)
    X = np.stack([t ** (2 * i + 1) for i in range(nterms)], 1) / f[:, None]
    one = np.ones_like(t)
    w = np.ones_like(t)
    for _ in range(iters):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(X * sw[:, None], one * sw, rcond=None)
        e = np.abs(X @ c - one)
        w = w * e
        w /= w.sum()
    return c.astype(np.float32)


def eval_f32(c, t):
    """The kernel's evaluation order in float32: Horner in s = t^2, then * t."""
    t = np.asarray(t, np.float32)
    s = (t * t).astype(np.float32)
    p = np.float32(c[-1])
    for k in range(len(c) - 2, -1, -1):
        p = (p * s + np.float32(c[k])).astype(np.float32)
    return (p * t).astype(np.float32)


def main():
    c = fit()
    t = np.concatenate([np.logspace(-8, 0, 100001), np.linspace(0, 1, 200001)[1:]]).astype(np.float32)
    ref = np.arctan(t.astype(np.float64))
    r = eval_f32(c, t).astype(np.float64)
    print("coefficients (t^1 .. t^%d):" % (2 * len(c) - 1))
    print("  " + ", ".join("%.9ef" % x for x in c))
    print("float32 relative error %.3e, absolute %.3e" % (np.max(np.abs(r - ref) / ref), np.max(np.abs(r - ref))))


if __name__ == "__main__":
    main()
