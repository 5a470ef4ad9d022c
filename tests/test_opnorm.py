"""Power-iteration operator-norm estimate (getopnorm, matlab/getopnorm.m:1-17).

CPU: the oracle's K^H is the adjoint of its K under the solver's inner
products, its normal operator is Hermitian, and the power iteration reaches
the largest eigenvalue of the dense normal matrix on tiny problems (the
reference holds no golden value for the estimate; these pin the oracle to its
definition).  GPU: avx_operator_opnorm and avx_solver_opnorm against the
oracle from the same start vector (1e-5 relative: fp32 operator applications
against float64), the initial steps they set, and a run from those steps
against the oracle's run from its own estimate (1e-4 relative L2 image error).
"""

import numpy as np
import pytest

from oracle import opnorm as on
from oracle import radial as rd
from oracle import solvers as so
from oracle.cartesian import CartesianOperator as OCart

METHODS = ["TV", "TVTEMP", "TGV2", "ICTV", "ICTGV2"]
REL_EST = 1e-5
REL_IMG = 1e-4


def cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _lines_mask(rng, T, H, W, frac=3):
    m = np.zeros((T, H, W))
    for t in range(T):
        m[t, rng.choice(H, size=max(1, H // frac), replace=False), :] = 1
    return m


def _small_problem(seed, W=10, H=8, C=2, T=3):
    rng = np.random.default_rng(seed)
    mask = _lines_mask(rng, T, H, W)
    b1 = cplx(rng, (C, H, W))
    b1 /= np.sqrt(np.sum(np.abs(b1) ** 2, axis=0, keepdims=True))
    return OCart(W, H, C, T, mask=mask, centered=True), b1, rng


@pytest.mark.parametrize("method", METHODS)
def test_oracle_adjoint(method):
    """<K x, (d, z)> = <x, K^H (d, z)> with the dual inner product that
    counts the symmetrised gradient's off-diagonal entries twice."""
    op, b1, rng = _small_problem(1)
    p = so.init_params(method)
    K, Kh, P = on.method_operator(method, op, b1, p)
    T, H, W = op.T, op.H, op.W
    x = [cplx(rng, (T, H, W)) for _ in range(P)]
    d0, z0 = K(x)
    d = [cplx(rng, c.shape) for c in d0]
    z = cplx(rng, z0.shape)
    lhs = on.dual_dot(method, d0, d) + np.vdot(z0, z)
    xh = Kh(d, z)
    rhs = sum(np.vdot(a, b) for a, b in zip(x, xh))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def _dense_normal(normal, P, shape):
    n = int(np.prod(shape))
    M = np.zeros((P * n, P * n), complex)
    for j in range(P * n):
        e = np.zeros(P * n, complex)
        e[j] = 1.0
        y = normal([e[c * n:(c + 1) * n].reshape(shape) for c in range(P)])
        M[:, j] = np.concatenate([c.ravel() for c in y])
    return M


@pytest.mark.parametrize("method", ["ENCODING", "TV", "TGV2", "ICTV"])
def test_oracle_reaches_largest_eigenvalue(method):
    op, b1, rng = _small_problem(2, W=6, H=5, C=2, T=3)
    shape = (op.T, op.H, op.W)
    if method == "ENCODING":
        normal, P = on.encoding_normal(op, b1), 1
    else:
        p = so.init_params(method)
        normal, P = on.method_normal(method, op, b1, p), on.method_operator(method, op, b1, p)[2]
    M = _dense_normal(normal, P, shape)
    assert np.linalg.norm(M - M.conj().T) < 1e-12 * np.linalg.norm(M)
    lam = np.linalg.eigvalsh(M).max()
    x0 = [cplx(rng, shape)] + [cplx(rng, shape) for _ in range(P - 1)]
    est10 = on.getopnorm(normal, x0, 10)
    est = on.getopnorm(normal, x0, 5000)
    assert est10 <= lam * (1 + 1e-12)
    assert lam * (1 - 1e-6) <= est <= lam * (1 + 1e-12)


def test_oracle_rejects_zero_iterations():
    op, b1, rng = _small_problem(3)
    with pytest.raises(ValueError):
        on.getopnorm(on.encoding_normal(op, b1), [cplx(rng, (op.T, op.H, op.W))], 0)


def test_steps_form():
    s, t = on.opnorm_steps(9.0, 2.0)
    assert np.isclose(s, 2.0 / 3.0) and np.isclose(t, 1.0 / 6.0)
    assert np.isclose(s * t * 9.0, 1.0)


# ---------------------------------------------------------------------------
# device
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def _rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.gpu
@pytest.mark.parametrize("dft", [0, 1])
@pytest.mark.parametrize("W,H,C,T,centered", [(32, 24, 4, 5, False), (64, 64, 3, 4, True)])
def test_encoding_opnorm_matches_oracle(av, W, H, C, T, centered, dft):
    rng = np.random.default_rng(W + C)
    mask = _lines_mask(rng, T, H, W)
    b1 = cplx(rng, (C, H, W)).astype(np.complex64)
    x0 = cplx(rng, (T, H, W)).astype(np.complex64)
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(mask.astype(np.float32)), centered=centered)
    op.dft_mode = dft
    est, hist = op.opnorm(av.to_device(x0), av.to_device(b1), 10, history=True)
    oop = OCart(W, H, C, T, mask=mask, centered=centered)
    oh = []
    ref = on.getopnorm(on.encoding_normal(oop, b1.astype(complex)), [x0.astype(complex)], 10, oh)
    assert _rel(est, ref) < REL_EST, (est, ref)
    assert np.allclose(hist, oh, rtol=REL_EST)


@pytest.mark.gpu
def test_encoding_opnorm_radial_matches_oracle(av):
    W, H, C, T, nfe, spf, osf = 24, 20, 3, 3, 48, 9, 1.5
    rng = np.random.default_rng(4)
    traj, dens = rd.golden_angle_radial(nfe, spf, T)
    traj, dens = traj.astype(np.float32), dens.astype(np.float32)
    b1 = cplx(rng, (C, H, W)).astype(np.complex64)
    x0 = cplx(rng, (T, H, W)).astype(np.complex64)
    g = av.RadialOperator(W, H, C, T, av.to_device(traj), av.to_device(dens), spf, 3.0, 8.0, osf)
    o = rd.RadialOperator(W, H, C, T, traj.astype(float), dens.astype(float), 3.0, 8.0, osf)
    est = g.opnorm(av.to_device(x0), av.to_device(b1), 10)
    ref = on.getopnorm(on.encoding_normal(o, b1.astype(complex)), [x0.astype(complex)], 10)
    assert _rel(est, ref) < REL_EST, (est, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["TV", "TGV2", "ICTGV2"])
def test_solver_opnorm_radial_matches_oracle(av, method):
    """The whole primal-dual operator with the gridding operator as its
    encoding part."""
    W, H, C, T, nfe, spf, osf = 24, 20, 3, 3, 48, 9, 1.5
    rng = np.random.default_rng(8)
    traj, dens = rd.golden_angle_radial(nfe, spf, T)
    traj, dens = traj.astype(np.float32), dens.astype(np.float32)
    b1 = cplx(rng, (C, H, W)).astype(np.complex64)
    x0 = cplx(rng, (T, H, W)).astype(np.complex64)
    g = av.RadialOperator(W, H, C, T, av.to_device(traj), av.to_device(dens), spf, 3.0, 8.0, osf)
    o = rd.RadialOperator(W, H, C, T, traj.astype(float), dens.astype(float), 3.0, 8.0, osf)
    s = av.Solver(method, g)
    est = s.opnorm(av.to_device(x0), av.to_device(b1), 10)
    p = so.init_params(method)
    ref = on.getopnorm(on.method_normal(method, o, b1.astype(complex), p), on.method_start(method, x0), 10)
    assert _rel(est, ref) < REL_EST, (est, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("dft", [0, 1])
@pytest.mark.parametrize("method", METHODS)
def test_solver_opnorm_matches_oracle(av, method, dft):
    from avionic_b200 import synth
    prob = synth.small(11)
    T, C, H, W = prob["kdata"].shape
    rng = np.random.default_rng(5)
    x0 = cplx(rng, (T, H, W)).astype(np.complex64)
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    op.dft_mode = dft
    s = av.Solver(method, op)
    ratio = s.params.sigmaTauRatio
    est, hist = s.opnorm(av.to_device(x0), av.to_device(prob["b1"]), 10, set_steps=True, history=True)
    oop = OCart(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params(method)
    oh = []
    ref = on.getopnorm(on.method_normal(method, oop, prob["b1"].astype(complex), p),
                       on.method_start(method, x0), 10, oh)
    assert _rel(est, ref) < REL_EST, (est, ref)
    assert np.allclose(hist, oh, rtol=REL_EST)
    sig, tau = on.opnorm_steps(ref, ratio)
    assert _rel(s.params.sigma, sig) < REL_EST and _rel(s.params.tau, tau) < REL_EST


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["TGV2", "ICTGV2"])
def test_run_from_opnorm_steps_matches_oracle(av, method):
    """A reconstruction started from the estimated steps equals the oracle's
    reconstruction started from its own estimate."""
    import torch
    from avionic_b200 import synth
    prob = synth.small(7)
    T, C, H, W = prob["kdata"].shape
    rng = np.random.default_rng(6)
    x0 = cplx(rng, (T, H, W)).astype(np.complex64)
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    s = av.Solver(method, op)
    p = s.params
    p.maxIt = 150
    s.params = p
    s.opnorm(av.to_device(x0), av.to_device(prob["b1"]), 10, set_steps=True)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))

    oop = OCart(W, H, C, T, mask=prob["mask"], centered=False)
    po = so.init_params(method)
    po.lam = oop.adapt_lambda(*po.adapt_kd)
    po.maxIt = 150
    ref = on.getopnorm(on.method_normal(method, oop, prob["b1"].astype(complex), po),
                       on.method_start(method, x0), 10)
    po.sigma, po.tau = on.opnorm_steps(ref, po.sigmaTauRatio)
    xo = so.run(method, prob["kdata"].astype(complex), np.zeros((T, H, W), complex),
                prob["b1"].astype(complex), oop, po)
    r = float(np.linalg.norm((x.cpu().numpy() - xo).ravel()) / np.linalg.norm(xo.ravel()))
    assert r < REL_IMG, r
