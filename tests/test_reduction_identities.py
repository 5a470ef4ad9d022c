"""ICTV and TVtemp pinned by independent restatements.

The reference holds no known answers for ICTV (CUDA/src/ictv.cpp:202-370) or
TVtemp (CUDA/src/tv_temp.cpp:95-182).  Beyond the oracle's line-by-line
restatement (oracle/solvers.py), two restatements written differently check
both the oracle and the CUDA path:

* ICTV as a generic primal-dual loop over the stacked operator
  K_reg = [[G1, -G1], [0, G2]] built as sparse matrices (G = the weighted
  forward-difference gradient, zero at the last index), with the reference's
  loop order, proximal radii and step rule (whose norm of K e covers the data
  term alone, ictv.cpp:97-128);
* TVtemp with a full mask, one coil and b1 = 1, where K is the unitary 2D
  transform: the loop then equals, exactly, a temporal-TV denoising of
  f = K^H d run pixel by pixel along t in the image domain (K^H K = I).

The oracle matches both to 1e-10; the device to 1e-4 (the reconstruction
tolerance).
"""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import solvers as so
from oracle import stencils as st
from oracle.cartesian import CartesianOperator

REL_IMG = 1e-4


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _fwd_diff(n):
    """(D u)_i = u_{i+1} - u_i, 0 at the last index."""
    d = sp.lil_matrix((n, n))
    for i in range(n - 1):
        d[i, i] = -1.0
        d[i, i + 1] = 1.0
    return d.tocsr()


def _grad_mats(T, H, W, w):
    """Weighted gradient of a (T, H, W) array flattened in C order."""
    It, Ih, Iw = sp.identity(T), sp.identity(H), sp.identity(W)
    dx = sp.kron(sp.kron(It, Ih), _fwd_diff(W)) / w[0]
    dy = sp.kron(sp.kron(It, _fwd_diff(H)), Iw) / w[1]
    dtm = sp.kron(sp.kron(_fwd_diff(T), Ih), Iw) / w[2]
    return [dx.tocsr(), dy.tocsr(), dtm.tocsr()]


def _prox_ball(ys, radius):
    """Pointwise projection of the vector field ys onto the ball of `radius`."""
    n = np.sqrt(sum(np.abs(y) ** 2 for y in ys))
    d = np.maximum(1.0, n / radius)
    return [y / d for y in ys]


def ictv_matrix_loop(data, b1, mask, p, iters):
    """ICTV by stacked sparse operators (see the module docstring)."""
    T, C, H, W = data.shape
    op = CartesianOperator(W, H, C, T, mask=mask, centered=False)
    w1 = (st.time_space_weights(p.timeSpaceWeight)[0],) * 2 + (st.time_space_weights(p.timeSpaceWeight)[1],)
    w2 = (st.time_space_weights(p.timeSpaceWeight2)[0],) * 2 + (st.time_space_weights(p.timeSpaceWeight2)[1],)
    G1, G2 = _grad_mats(T, H, W, w1), _grad_mats(T, H, W, w2)
    n = T * H * W
    m = min(p.alpha, 1.0 - p.alpha)
    rad1, rad3 = p.alpha1 * (p.alpha / m), p.alpha1 * ((1.0 - p.alpha) / m)
    x1, x3 = np.zeros(n, complex), np.zeros(n, complex)
    e1, e3 = x1.copy(), x3.copy()
    y1 = [np.zeros(n, complex) for _ in range(3)]
    y3 = [np.zeros(n, complex) for _ in range(3)]
    z = np.zeros(data.shape, complex)
    sigma, tau = p.sigma, p.tau
    shape = (T, H, W)
    steps = []
    for k in range(iters):
        y1 = _prox_ball([y1[i] + sigma * (G1[i] @ (e1 - e3)) for i in range(3)], rad1)
        y3 = _prox_ball([y3[i] + sigma * (G2[i] @ e3) for i in range(3)], rad3)
        z = mask[:, None] * ((z + sigma * op.backward(e1.reshape(shape), b1) - sigma * data) / (1.0 + sigma / p.lam))
        khz = op.forward(z.copy(), b1).ravel()
        g1t = sum(G1[i].T @ y1[i] for i in range(3))   # = -div1
        g2t = sum(G2[i].T @ y3[i] for i in range(3))   # = -div3
        x1n = x1 - tau * (khz + g1t)
        x3n = x3 - tau * (-g1t + g2t)
        e1, e3 = 2.0 * x1n - x1, 2.0 * x3n - x3
        x1, x3 = x1n, x3n
        if k < 10 or k % 50 == 0:
            d1, d3 = e1 - x1, e3 - x3
            nKx = np.linalg.norm(op.backward(d1.reshape(shape), b1).ravel())
            nx = np.sqrt(np.linalg.norm(d1) ** 2 + np.linalg.norm(d3) ** 2)
            sigma, tau = st.step_rule(sigma, tau, nKx, nx, p.sigmaTauRatio)
        steps.append((sigma, tau))
    return x1.reshape(shape), steps


def tvtemp_pixelwise_loop(data, p, iters):
    """TVtemp with a full mask, one coil, b1 = 1: temporal-TV denoising of
    f = K^H d, pixel by pixel along t."""
    f = np.fft.fft2(data[:, 0], norm="ortho")  # k-space -> image (the operator's F^-1)
    T = f.shape[0]
    D = _fwd_diff(T) / p.dt
    X = f.reshape(T, -1) * 0.0
    E = X.copy()
    Y = np.zeros_like(X)
    Z = np.zeros_like(X)  # K^H z in the image domain
    F = f.reshape(T, -1)
    sigma, tau = p.sigma, p.tau
    for k in range(iters):
        Y = Y + sigma * (D @ E)
        Y = Y / np.maximum(1.0, np.abs(Y))
        Z = (Z + sigma * E - sigma * F) / (1.0 + sigma / p.lam)
        Xn = X - tau * (Z + D.T @ Y)
        E = 2.0 * Xn - X
        X = Xn
        if k < 10 or k % 50 == 0:
            dd = E - X
            nKx = np.sqrt(np.linalg.norm(D @ dd) ** 2 + np.linalg.norm(dd) ** 2)
            sigma, tau = st.step_rule(sigma, tau, nKx, np.linalg.norm(dd), p.sigmaTauRatio)
    return X.reshape(f.shape)


def _ictv_problem():
    from avionic_b200 import synth
    prob = synth.small(21, H=12, W=10, T=5, C=3, R=2)
    p = so.init_params("ICTV")
    p.lam, p.maxIt = 3.0, 80
    return prob, p


def _tvtemp_problem():
    rng = np.random.default_rng(31)
    T, H, W = 8, 9, 7
    base = rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))
    steps = np.where(np.arange(T) < T // 2, 0.0, 1.0)[:, None, None]
    x = base[None] * (1.0 + 0.5 * steps)
    x = x + 0.05 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    d = np.fft.ifft2(x, norm="ortho")[:, None].astype(np.complex64)  # image -> k-space, one coil, b1 = 1
    p = so.init_params("TVTEMP")
    p.lam, p.maxIt, p.dt = 2.0, 80, 1.0
    return d, p


def test_oracle_ictv_matches_the_matrix_restatement():
    prob, p = _ictv_problem()
    T, C, H, W = prob["kdata"].shape
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    tr = {}
    xo = so.ictv(prob["kdata"].astype(complex), np.zeros((T, H, W), complex), prob["b1"].astype(complex), op, p, tr)
    xm, steps = ictv_matrix_loop(prob["kdata"].astype(complex), prob["b1"].astype(complex),
                                 prob["mask"].astype(float), p, p.maxIt)
    assert rel(xo, xm) < 1e-10
    assert np.allclose(np.array(tr["steps"]), np.array(steps), rtol=1e-12)


def test_oracle_tvtemp_reduces_to_pixelwise_temporal_tv():
    d, p = _tvtemp_problem()
    T, C, H, W = d.shape
    op = CartesianOperator(W, H, C, T, mask=np.ones((T, H, W)), centered=False)
    xo = so.tvtemp(d.astype(complex), np.zeros((T, H, W), complex), np.ones((1, H, W), complex), op, p)
    xp = tvtemp_pixelwise_loop(d.astype(complex), p, p.maxIt)
    assert rel(xo, xp) < 1e-10


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


@pytest.mark.gpu
@pytest.mark.parametrize("dft", [0, 1], ids=["fp32", "split"])
def test_device_ictv_matches_the_matrix_restatement(av, dft):
    prob, p = _ictv_problem()
    T, C, H, W = prob["kdata"].shape
    xm, steps = ictv_matrix_loop(prob["kdata"].astype(complex), prob["b1"].astype(complex),
                                 prob["mask"].astype(float), p, p.maxIt)
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    op.dft_mode = dft
    q = av.default_params(av.ICTV)
    q.maxIt, q.lambda_, q.adaptLambda = p.maxIt, p.lam, 0
    s = av.Solver(av.ICTV, op, q)
    x = av.to_device(np.zeros((T, H, W), np.complex64))
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))
    assert rel(x.cpu().numpy(), xm) < REL_IMG
    assert abs(s.stats().sigma - steps[-1][0]) <= 1e-5 * steps[-1][0]


@pytest.mark.gpu
def test_device_tvtemp_reduces_to_pixelwise_temporal_tv(av):
    d, p = _tvtemp_problem()
    T, C, H, W = d.shape
    xp = tvtemp_pixelwise_loop(d.astype(complex), p, p.maxIt)
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(np.ones((T, H, W), np.float32)), centered=False)
    q = av.default_params(av.TVTEMP)
    q.maxIt, q.lambda_, q.adaptLambda, q.dt = p.maxIt, p.lam, 0, p.dt
    s = av.Solver(av.TVTEMP, op, q)
    x = av.to_device(np.zeros((T, H, W), np.complex64))
    s.run(av.to_device(d), x, av.to_device(np.ones((1, H, W), np.complex64)))
    assert rel(x.cpu().numpy(), xp) < REL_IMG
