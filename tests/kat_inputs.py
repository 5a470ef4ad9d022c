"""Input builders for the reference known-answer tests.

The reference's fixtures fill a vector with its own linear index
(CUDA/test/tv.cc:22-36, tgv2.cc:22-36, derivatives.cc:28-40) and slice it;
b1 is 1 for coil 0 and 2i for coil 1 (tv.cc:353-356).  These helpers build the
same inputs as numpy arrays in the (T, H, W) / (T, C, H, W) / (C, H, W)
layouts, shared by the oracle KAT tests and the GPU KAT tests.
"""

import numpy as np


def lin(n, start=0):
    return np.arange(start, start + n, dtype=np.float64).astype(np.complex128)


def image(W, H, T, start=0):
    return lin(W * H * T, start).reshape(T, H, W)


def kspace(W, H, C, T):
    return lin(W * H * C * T).reshape(T, C, H, W)


def b1_std(W, H, C, scales=None):
    """Coil maps: coil 1 scaled by 2i, others 1 (tv.cc:353-356), or real
    per-coil scales (cartesian_operator.cc:229-234)."""
    b1 = np.ones((C, H, W), dtype=np.complex128)
    if scales is None:
        if C > 1:
            b1[1] *= 2j
    else:
        for c, s in enumerate(scales):
            b1[c] *= s
    return b1


def mask_of(spec, W, H, T):
    if spec is None:
        return None
    if spec == "ones":
        return np.ones((T, H, W))
    raise ValueError(spec)


def at(arr, pos):
    """arr (T,H,W) at reference position [x, y, t]."""
    x, y, t = pos
    return arr[t, y, x]


def radial_fixture(k):
    """The radial operator's test fixture (CUDA/test/noncartesian_operator.cc:17-101):
    trajectory (T, 2, S) with sample cnt of spoke sp in frame f at
    kx = cnt / nFE - 0.5, ky = (f spf + sp) / nSpokes - 0.5 (horizontal spokes),
    density 1, and coil maps of constant value 1, 2, 3."""
    W, H, C, T = k["width"], k["height"], k["coils"], k["frames"]
    nfe, spf, nsp = k["nFE"], k["spokesPerFrame"], k["nSpokes"]
    S = nfe * spf
    traj = np.zeros((T, 2, S), dtype=np.float32)
    for f in range(T):
        for sp in range(spf):
            for cnt in range(nfe):
                traj[f, 0, sp * nfe + cnt] = np.float32(cnt / nfe) - np.float32(0.5)
                traj[f, 1, sp * nfe + cnt] = np.float32((f * spf + sp) / nsp) - np.float32(0.5)
    dens = np.ones((T, S), dtype=np.float32)
    b1 = np.stack([np.full((H, W), v, dtype=np.complex128) for v in k["b1_per_coil"]])
    return traj, dens, b1
