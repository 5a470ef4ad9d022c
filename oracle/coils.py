"""Variational H1 coil-sensitivity estimation, float64 (test infrastructure).

Restates CUDA/src/coil_construction.cpp (PerformCoilConstruction :447-556,
B1FromUH1 :363-445, UTGV2Recon :75-215, B1Recon :217-361, FindMaximumSum
:55-73) and CUDA/src/cartesian_coil_construction.cpp:23-86
(TimeAveragedReconstruction), with the defaults of InitParams (:22-48).

The H1 system (mu |u|^2 I - Laplace_periodic) b = mu u |crec_c| is solved
exactly (sparse LU); the reference runs AGILE's CG (<= 800 iterations,
tolerance 1e-12, coil_construction.cpp:378-411), whose converged result is the
same solution.  2D stencils are the (x, y) restriction of the 3D ones
(utils.cpp:156-181, 525-568, 817-844, 1078-1117): gradient (D+x, D+y),
symmetrised gradient (xx, yy, xy), their negative adjoints as divergences.
Arrays: coil images (C, H, W), single images (H, W).
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import stencils as st
from .cartesian import ifft2u


def default_params():
    """CoilConstruction::InitParams (coil_construction.cpp:22-48)."""
    return dict(uH1mu=1e-5, uReg=0.2, uNrIt=100, uSigma=np.sqrt(1.0 / 12.0), uTau=np.sqrt(1.0 / 12.0),
                uAlpha0=np.sqrt(2.0), uAlpha1=1.0, b1Reg=2.0, b1NrIt=500, b1Sigma=np.sqrt(1.0 / 8.0),
                b1Tau=np.sqrt(1.0 / 8.0), b1FinalReg=0.1, b1FinalNrIt=1000)


def _3(u):
    return u[None]


def grad2(u):
    g = st.gradient(_3(u))
    return [g[0][0], g[1][0]]


def div2(y):
    return st.divergence([_3(y[0]), _3(y[1]), np.zeros_like(_3(y[0]))])[0]


def symgrad2(v):
    z = np.zeros_like(_3(v[0]))
    e = st.sym_gradient([_3(v[0]), _3(v[1]), z])
    return [e[0][0], e[1][0], e[3][0]]


def symdiv2(w):
    z = np.zeros_like(_3(w[0]))
    d = st.sym_divergence([_3(w[0]), _3(w[1]), z, _3(w[2]), z, z])
    return [d[0][0], d[1][0]]


def prox2(y, scale):
    n = np.sqrt(np.abs(y[0]) ** 2 + np.abs(y[1]) ** 2)
    d = np.maximum(1.0, scale * n)
    return [c / d for c in y]


def prox2sym(y, scale):
    n = np.sqrt(np.abs(y[0]) ** 2 + np.abs(y[1]) ** 2 + 2.0 * np.abs(y[2]) ** 2)
    d = np.maximum(1.0, scale * n)
    return [c / d for c in y]


def laplace_periodic(u):
    """-(D-x D+x + D-y D+y) u with wrapped differences (cg_forward_operation.h:47-70)."""
    a = _3(u)
    gx = st.diff(a, 1, wrap=True)
    gy = st.diff(a, 2, wrap=True)
    return -(st.bdiff(gx, 1, wrap=True) + st.bdiff(gy, 2, wrap=True))[0]


def time_averaged_reconstruction(kdata, mask, centered=False, apply_phase=True):
    """CartesianCoilConstruction::TimeAveragedReconstruction
    (cartesian_coil_construction.cpp:23-86).  Returns (u (H,W), crec (C,H,W))."""
    data = np.sum(kdata, axis=0)
    m = np.maximum(np.sum(mask, axis=0), 1.0)
    crec = np.stack([ifft2u(data[c] / m, centered) for c in range(data.shape[0])])
    u = np.sqrt(np.sum(np.abs(crec) ** 2, axis=0)).astype(complex)
    if apply_phase:
        u = u * np.exp(1j * np.angle(np.sum(crec, axis=0)))
    return u, crec


def _h1_matrix(mu_u, H, W):
    n = H * W
    idx = np.arange(n).reshape(H, W)
    rows, cols, vals = [], [], []
    for (dy, dx) in ((0, 1), (0, -1), (1, 0), (-1, 0)):
        nb = np.roll(np.roll(idx, -dy, axis=0), -dx, axis=1)
        rows.append(idx.ravel())
        cols.append(nb.ravel())
        vals.append(-np.ones(n))
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(4.0 + mu_u.ravel())
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def b1_from_u_h1(u, crec, p):
    """CoilConstruction::B1FromUH1 (coil_construction.cpp:363-445): |b1| per coil."""
    C, H, W = crec.shape
    crec_real = p["uH1mu"] * np.abs(crec)
    mu_u = p["uH1mu"] * np.abs(u) ** 2
    A = _h1_matrix(mu_u, H, W)
    lu = spla.splu(A)
    b1 = np.zeros((C, H, W), complex)
    for c in range(C):
        y = np.conj(u) * crec_real[c]
        b1[c] = (lu.solve(np.real(y).ravel()) + 1j * lu.solve(np.imag(y).ravel())).reshape(H, W)
    nrm = np.sqrt(np.sum(np.abs(b1) ** 2, axis=0))
    b1 = b1 / nrm
    return np.abs(b1).astype(complex)


def find_maximum_sum(crec):
    """FindMaximumSum (coil_construction.cpp:55-73): coil with the largest sum |crec|."""
    return int(np.argmax([np.sum(np.abs(c)) for c in crec]))


def utgv2_recon(b10, crec0, x1, inds, p):
    """UTGV2Recon (coil_construction.cpp:75-215): 2D TGV2 estimate of the image
    from the coils in inds; x1 (H,W) is the initial value; returns the result."""
    nu = p["uReg"]
    sig, tau = p["uSigma"], p["uTau"]
    x1 = x1.astype(complex).copy()
    ext1 = x1.copy()
    x2 = [np.zeros_like(x1), np.zeros_like(x1)]
    ext2 = [np.zeros_like(x1), np.zeros_like(x1)]
    y1 = [np.zeros_like(x1), np.zeros_like(x1)]
    y2 = [np.zeros_like(x1) for _ in range(3)]
    Lw = np.zeros_like(x1)
    sumB1 = np.zeros_like(x1)
    for c in inds:
        Lw = Lw + np.conj(b10[c]) * crec0[c]
        sumB1 = sumB1 + np.conj(b10[c]) * b10[c]
    Ib = 1.0 / (1.0 + tau * sumB1)
    for _ in range(int(p["uNrIt"])):
        g = grad2(ext1)
        y1 = [y1[i] + sig * (g[i] - ext2[i]) for i in range(2)]
        e = symgrad2(ext2)
        y2 = [y2[i] + sig * e[i] for i in range(3)]
        y1 = prox2(y1, 1.0 / (p["uAlpha1"] * nu))
        y2 = prox2sym(y2, 1.0 / (p["uAlpha0"] * nu))
        n1 = x1 + tau * div2(y1)
        sd = symdiv2(y2)
        n2 = [x2[i] + tau * (y1[i] + sd[i]) for i in range(2)]
        n1 = (n1 + tau * Lw) * Ib
        ext1 = 2.0 * n1 - x1
        ext2 = [2.0 * n2[i] - x2[i] for i in range(2)]
        x1, x2 = n1, n2
    return x1


def b1_recon(u0, crec, coils, max_it, mu, p):
    """B1Recon (coil_construction.cpp:217-361): H1-regularised coil maps for
    image u0 (H,W) and coil images crec (coils,H,W); returns (coils,H,W)
    normalised so that sum_c |b1_c|^2 = 1."""
    sig, tau = p["b1Sigma"], p["b1Tau"]
    un = u0 / np.max(np.abs(u0))
    sumU = 1.0 + tau * np.abs(un) ** 2
    Lw = np.conj(un)[None] * crec[:coils]
    Iu = 1.0 / sumU
    x1 = np.zeros((coils,) + u0.shape, complex)
    ext1 = x1.copy()
    y = [np.zeros_like(x1), np.zeros_like(x1)]
    for _ in range(int(max_it)):
        for c in range(coils):
            g = grad2(ext1[c])
            for k in range(2):
                y[k][c] = (y[k][c] + sig * g[k]) * (1.0 / (1.0 + sig / mu))
        n1 = np.stack([x1[c] + tau * div2([y[0][c], y[1][c]]) for c in range(coils)])
        n1 = (n1 + tau * Lw) * Iu[None]
        ext1 = 2.0 * n1 - x1
        x1 = n1
    nrm = np.sqrt(np.sum(np.abs(x1) ** 2, axis=0))
    return x1 / nrm[None]


def time_averaged_radial(kdata, traj, dens, W, H, apply_phase=True):
    """NoncartesianCoilConstruction::TimeAveragedReconstruction
    (noncartesian_coil_construction.cpp:21-127): all frames' samples through
    one gridding adjoint (kernel width 3, sector width 8, osf 2) per coil,
    with the gridding of oracle/radial.py.  kdata (T,C,S)."""
    from .radial import RadialOperator
    T, C, S = kdata.shape
    tr = np.concatenate([traj[f] for f in range(T)], axis=1)[None]      # (1, 2, T S)
    de = dens.reshape(1, T * S)
    op = RadialOperator(W, H, 1, 1, tr, de, 3.0, 8.0, 2.0)
    ones = np.ones((1, H, W), complex)
    crec = np.stack([op.forward(kdata[:, c, :].reshape(1, 1, T * S), ones)[0] for c in range(C)])
    u = np.sqrt(np.sum(np.abs(crec) ** 2, axis=0)).astype(complex)
    if apply_phase:
        u = u * np.exp(1j * np.angle(np.sum(crec, axis=0)))
    return u, crec


def perform_coil_construction(kdata, mask, p=None, centered=False):
    """PerformCoilConstruction (coil_construction.cpp:447-556).  Returns
    (u (C,H,W) the sequence of image estimates, b1 (C,H,W))."""
    u0, crec = time_averaged_reconstruction(kdata, mask, centered)
    return estimate_from(u0, crec, p)


def estimate_from(u0, crec, p=None):
    """The part of PerformCoilConstruction after the time average."""
    p = p or default_params()
    C = crec.shape[0]
    u0 = np.abs(u0).astype(complex)
    absb1 = b1_from_u_h1(u0, crec, p)
    H, W = u0.shape
    b1 = np.zeros((C, H, W), complex)
    u = np.zeros((C, H, W), complex)
    inds = [find_maximum_sum(crec)]
    b1[inds[0]] = absb1[inds[0]]
    u[0] = utgv2_recon(b1, crec, np.zeros((H, W), complex), inds, p)
    w = np.zeros((H, W), complex)
    uMax = u[0]
    for cnt in range(1, C):
        b = absb1[inds[cnt - 1]]
        w = np.sqrt(w * w + np.conj(b) * b)
        a1 = np.abs(crec[inds[cnt - 1]])
        best, max_ind = -np.inf, -1
        for k in range(C):
            if k in inds:
                continue
            v = np.sum(a1 * np.abs(crec[k]))
            if v > best:
                best, max_ind = v, k
        inds.append(max_ind)
        u_in = absb1[max_ind] * u[cnt - 1] * w
        crec_in = crec[max_ind] * w
        x1 = b1_recon(u_in, crec_in[None], 1, p["b1NrIt"], p["b1Reg"], p)[0]
        b1[max_ind] = absb1[max_ind] * np.exp(1j * np.angle(x1))
        uMax = utgv2_recon(b1, crec, u[cnt - 1], inds, p)
        u[cnt] = uMax
    b1 = b1_recon(uMax, crec, C, p["b1FinalNrIt"], p["b1FinalReg"], p)
    return u, b1
