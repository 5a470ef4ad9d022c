"""Pin the float64 oracle against the reference's own known-answer tests.

Every expected value comes from the reference gtest suite (CUDA/test/*.cc,
transcribed in tests/golden/reference_kats.json with file:line); the
derivative KATs are restated from CUDA/test/derivatives.cc:169-650 as the
integer formulas the reference asserts.  Tolerance is the reference's own
1e-3 absolute (CUDA/test/test_utils.h:11) except where noted.
"""

import numpy as np
import pytest

from oracle import stencils as st
from oracle import solvers as so
from oracle.cartesian import CartesianOperator, fft2u, ifft2u
from tests import kat_inputs as ki

EPS = 1e-3


# ---------------------------------------------------------------------------
# derivatives.cc: integer-exact boundary semantics
# ---------------------------------------------------------------------------

PARAMS = [(5, 5, 3), (4, 4, 3), (7, 5, 3), (5, 7, 3)]  # derivatives.cc:70-87


def _lin3(cols, rows, slices):
    return np.arange(cols * rows * slices, dtype=np.float64).reshape(slices, rows, cols)


def _L(x, y, z, cols, rows):
    return x + cols * (y + z * rows)


@pytest.mark.parametrize("cols,rows,slices", PARAMS)
@pytest.mark.parametrize("wrap", [False, True])
def test_derivatives_x(cols, rows, slices, wrap):
    a = _lin3(cols, rows, slices)
    L = lambda x, y, z: _L(x, y, z, cols, rows)  # noqa: E731
    d = st.diff(a, 1, wrap).ravel()
    assert d[L(0, 0, 0)] == 1 and d[L(2, 0, 1)] == 1
    if wrap:
        assert d[L(cols - 1, 0, 0)] == -cols + 1
        assert d[L(cols - 1, 0, slices - 1)] == -cols + 1
    else:
        assert d[L(cols - 1, 0, 0)] == 0 and d[L(cols - 1, 0, slices - 1)] == 0
    d = st.diff_t(a, 1, wrap).ravel()
    assert d[L(2, 0, 1)] == -1
    if wrap:
        assert d[L(cols - 1, 0, slices - 1)] == -1
        assert d[L(0, 0, 0)] == cols - 1
        assert d[L(cols - 1, 0, 0)] == -1
    else:
        assert d[L(cols - 1, 0, slices - 1)] == L(cols - 1, 0, slices - 1) - 1
        assert d[L(0, 0, 0)] == 0
        assert d[L(cols - 1, 0, 0)] == L(cols - 1, 0, 0) - 1
    d = st.bdiff(a, 1, wrap).ravel()
    assert d[L(1, 0, 0)] == 1
    if wrap:
        assert d[L(0, 0, 0)] == -cols + 1 and d[L(cols - 1, 0, 0)] == 1
    else:
        assert d[L(0, 0, 0)] == 0 and d[L(cols - 1, 0, 0)] == -cols + 2
    d = st.bdiff_t(a, 1, wrap).ravel()
    assert d[L(0, 0, 0)] == -1 and d[L(2, 0, 1)] == -1
    if wrap:
        assert d[L(cols - 1, 0, 0)] == cols - 1
        assert d[L(cols - 1, 0, slices - 1)] == cols - 1
    else:
        assert d[L(cols - 1, 0, 0)] == 0 and d[L(cols - 1, 0, slices - 1)] == 0


@pytest.mark.parametrize("cols,rows,slices", PARAMS)
@pytest.mark.parametrize("wrap", [False, True])
def test_derivatives_y(cols, rows, slices, wrap):
    a = _lin3(cols, rows, slices)
    m = a.ravel()
    L = lambda x, y, z: _L(x, y, z, cols, rows)  # noqa: E731
    d = st.diff(a, 2, wrap).ravel()
    assert d[L(0, 0, 0)] == cols and d[L(2, 0, 1)] == cols
    if wrap:
        assert d[L(0, rows - 1, 0)] == -cols * (rows - 1)
        assert d[L(0, rows - 1, slices - 1)] == -cols * (rows - 1)
    else:
        assert d[L(0, rows - 1, 0)] == 0 and d[L(0, rows - 1, slices - 1)] == 0
    d = st.diff_t(a, 2, wrap).ravel()
    if wrap:
        assert d[L(0, rows - 1, 0)] == -cols
        assert d[L(0, rows - 1, slices - 1)] == -cols
        assert d[L(0, 0, 0)] == cols * (rows - 1)
        assert d[L(2, 0, 1)] == cols * (rows - 1)
    else:
        assert d[L(0, rows - 1, 0)] == m[L(0, rows - 2, 0)]
        assert d[L(0, rows - 1, slices - 1)] == m[L(0, rows - 2, slices - 1)]
        assert d[L(0, 0, 0)] == 0
        assert d[L(2, 0, 1)] == -m[L(2, 0, 1)]
    d = st.bdiff(a, 2, wrap).ravel()
    if wrap:
        assert d[L(0, rows - 1, 0)] == cols
        assert d[L(0, rows - 1, slices - 1)] == cols
        assert d[L(0, 0, 0)] == -cols * (rows - 1)
        assert d[L(2, 0, 1)] == -cols * (rows - 1)
    else:
        assert d[L(0, rows - 1, 0)] == -m[L(0, rows - 2, 0)]
        assert d[L(0, rows - 1, slices - 1)] == -m[L(0, rows - 2, slices - 1)]
        assert d[L(0, 0, 0)] == 0
        assert d[L(2, 0, 1)] == m[L(2, 0, 1)]
    d = st.bdiff_t(a, 2, wrap).ravel()
    assert d[L(0, 0, 0)] == -cols and d[L(2, 0, 1)] == -cols
    if wrap:
        assert d[L(0, rows - 1, 0)] == cols * (rows - 1)
        assert d[L(0, rows - 1, slices - 1)] == cols * (rows - 1)
    else:
        assert d[L(0, rows - 1, 0)] == 0 and d[L(0, rows - 1, slices - 1)] == 0


@pytest.mark.parametrize("cols,rows,slices", PARAMS)
@pytest.mark.parametrize("wrap", [False, True])
def test_derivatives_t(cols, rows, slices, wrap):
    a = _lin3(cols, rows, slices)
    m = a.ravel()
    L = lambda x, y, z: _L(x, y, z, cols, rows)  # noqa: E731
    S = slices
    d = st.diff(a, 3, wrap).ravel()
    for p in [(0, 0, 0), (2, 1, 0), (0, rows - 1, 0)]:
        assert d[L(*p)] == rows * cols
    if wrap:
        assert d[L(0, 0, S - 1)] == -cols * rows * (S - 1)
        assert d[L(0, rows - 1, S - 1)] == -cols * rows * (S - 1)
    else:
        assert d[L(0, 0, S - 1)] == 0 and d[L(0, rows - 1, S - 1)] == 0
    d = st.diff_t(a, 3, wrap).ravel()
    if wrap:
        assert d[L(0, 0, S - 1)] == -cols * rows
        assert d[L(0, 0, 0)] == rows * cols * (S - 1)
        assert d[L(2, 1, 0)] == rows * cols * (S - 1)
        assert d[L(0, rows - 1, 0)] == rows * cols * (S - 1)
        assert d[L(0, rows - 1, S - 1)] == -cols * rows
    else:
        assert d[L(0, 0, S - 1)] == m[L(0, 0, S - 2)]
        assert d[L(0, 0, 0)] == 0
        assert d[L(2, 1, 0)] == -m[L(2, 1, 0)]
        assert d[L(0, rows - 1, 0)] == -m[L(0, rows - 1, 0)]
        assert d[L(0, rows - 1, S - 1)] == m[L(0, rows - 1, S - 2)]
    d = st.bdiff(a, 3, wrap).ravel()
    if wrap:
        assert d[L(0, 0, S - 1)] == cols * rows
        assert d[L(0, 0, 0)] == -rows * cols * (S - 1)
        assert d[L(2, 1, 0)] == -rows * cols * (S - 1)
        assert d[L(0, rows - 1, 0)] == -rows * cols * (S - 1)
        assert d[L(0, rows - 1, S - 1)] == cols * rows
    else:
        assert d[L(0, 0, S - 1)] == -m[L(0, 0, S - 2)]
        assert d[L(0, 0, 0)] == 0
        assert d[L(2, 1, 0)] == m[L(2, 1, 0)]
        assert d[L(0, rows - 1, 0)] == m[L(0, rows - 1, 0)]
        assert d[L(0, rows - 1, S - 1)] == -m[L(0, rows - 1, S - 2)]
    d = st.bdiff_t(a, 3, wrap).ravel()
    for p in [(0, 0, 0), (2, 1, 0), (0, rows - 1, 0)]:
        assert d[L(*p)] == -rows * cols
    if wrap:
        assert d[L(0, 0, S - 1)] == cols * rows * (S - 1)
        assert d[L(0, rows - 1, S - 1)] == cols * rows * (S - 1)
    else:
        assert d[L(0, 0, S - 1)] == 0 and d[L(0, rows - 1, S - 1)] == 0


@pytest.mark.parametrize("cols,rows,slices", PARAMS)
def test_derivatives_adjoint_pairs(cols, rows, slices):
    """<D u, v> = <u, D^T v> for every pair (the property derivatives.cc's
    Divergence / BackwardDivergence tests rely on, :282-416)."""
    rng = np.random.default_rng(7)
    u = rng.standard_normal((slices, rows, cols))
    v = rng.standard_normal((slices, rows, cols))
    for dim in (1, 2, 3):
        for wrap in (False, True):
            assert abs(np.vdot(st.diff(u, dim, wrap), v) - np.vdot(u, st.diff_t(v, dim, wrap))) < 1e-9
            assert abs(np.vdot(st.bdiff(u, dim, wrap), v) - np.vdot(u, st.bdiff_t(v, dim, wrap))) < 1e-9


# ---------------------------------------------------------------------------
# utils.cc, fft.cc
# ---------------------------------------------------------------------------

def test_ellipke(kats):
    for m, want in kats["ellipke"]["cases"]:
        assert abs(st.ellipke(m) - want) < EPS
    with pytest.raises(ValueError):
        st.ellipke(1.5)


def test_fft_centered_magnitudes(kats):
    a = np.arange(100, dtype=np.float64).reshape(10, 10).astype(complex)
    k = fft2u(a, centered=True)
    for (x, y), want in kats["fft_centered_10x10"]["values"]:
        assert abs(abs(k[y, x]) - want) < EPS
    back = ifft2u(k, centered=True)
    assert np.max(np.abs(back - a)) < 1e-9


# ---------------------------------------------------------------------------
# tv.cc
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name", ["tv_gradient_norm", "tv_scaled_gradient_norm"])
def test_tv_gradient_norms(kats, name):
    k = kats[name]
    W, H, T = k["dims"]
    n = st.norm3(st.gradient(ki.image(W, H, T), *k["w"]))
    for pos, want in k["values"]:
        assert abs(ki.at(n, pos) - want) < EPS


def test_tv_divergence_of_prox(kats):
    k = kats["tv_divergence_of_prox"]
    W, H, T = k["dims"]
    g = st.prox3(st.gradient(ki.image(W, H, T)), 1.0)
    d = st.divergence(g)
    for pos, want in k["values"]:
        assert abs(ki.at(d, pos).real - want) < EPS


def test_tv_adapt_lambda(kats):
    k = kats["tv_adapt_lambda"]
    W, H, T = k["dims"]
    op = CartesianOperator(W, H, k["coils"], T, mask=np.ones((T, H, W)))
    assert abs(op.adapt_lambda(k["k"], k["d"]) - k["value"]) < EPS


def test_tv_adapt_step(kats):
    k = kats["tv_adapt_step"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=ki.mask_of(k["mask"], W, H, T), centered=k["centered"])
    p = so.Params(sigma=k["sigma0"], tau=k["tau0"])
    b1 = ki.b1_std(W, H, C)
    so.tv_adapt_step(p, op, 1j * ki.image(W, H, T), b1, (1.0, 1.0, 1.0))
    assert abs(p.sigma - k["sigma"]) < EPS and abs(p.tau - k["tau"]) < EPS


def test_tv_norm(kats):
    k = kats["tv_norm"]
    W, H, T = k["dims"]
    for case in k["cases"]:
        s = complex(case["scale"]) if isinstance(case["scale"], str) else case["scale"]
        v = st.tv_norm(s * ki.image(W, H, T), *case["w"])
        assert abs(v - case["value"]) < EPS * max(1.0, 1e-3 * case["value"])


def _gap_setup(k):
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=ki.mask_of(k["mask"], W, H, T), centered=k["centered"])
    d = ki.kspace(W, H, C, T)
    z = np.full_like(d, k["z"])
    return W, H, T, C, op, d, z, so.Params(lam=k["lambda"])


# G*/gap goldens are FP32 sums of ~1e6: compare at 2e-6 relative, the FP32
# resolution of the printed value (CUDA/test/tv.cc:376, :435).
REL_GAP = 2e-6


def test_tv_gstar_and_gap(kats):
    for name in ("tv_gstar", "tv_pdgap"):
        k = kats[name]
        W, H, T, C, op, d, z, p = _gap_setup(k)
        x = ki.image(W, H, T)
        y = [np.zeros_like(x) for _ in range(3)]
        b1 = ki.b1_std(W, H, C)
        w = (1.0, 1.0, 1.0)
        if name == "tv_gstar":
            v = so.tv_gstar(p, op, x, y, z, d, b1, w)
        else:
            v = so.tv_gap(p, op, x, y, z, d, b1, w)
        assert abs(v - k["value"]) / k["value"] < REL_GAP, (name, v)


def test_tv_iteration(kats):
    k = kats["tv_iteration"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=None, centered=k["centered"])
    p = so.init_params("TV")
    p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = k["maxIt"]
    x = so.tv(ki.kspace(W, H, C, T), np.zeros((T, H, W), complex), ki.b1_std(W, H, C), op, p)
    for pos, want in k["values"]:
        assert abs(abs(ki.at(x, pos)) - want) < EPS, (pos, abs(ki.at(x, pos)), want)


# ---------------------------------------------------------------------------
# tgv2.cc
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name", ["tgv2_gradient_norms", "tgv2_scaled_gradient_norms"])
def test_tgv2_norm_fields(kats, name):
    k = kats[name]
    W, H, T = k["dims"]
    N = W * H * T
    A = ki.image(W, H, T)
    B = [ki.image(W, H, T, start=(i + 1) * N) for i in range(3)]
    g = st.gradient(A, *k["w"])
    n3 = st.norm3([g[i] - B[i] for i in range(3)])
    n6 = st.norm6(st.sym_gradient(B, *k["w"]))
    for pos, want in k["grad"]:
        assert abs(ki.at(n3, pos) - want) < EPS
    for pos, want in k["sym"]:
        assert abs(ki.at(n6, pos) - want) < EPS


def test_tgv2_sym_divergence_of_prox(kats):
    k = kats["tgv2_sym_divergence_of_prox"]
    W, H, T = k["dims"]
    N = W * H * T
    B = [ki.image(W, H, T, start=(i + 1) * N) for i in range(3)]
    y2 = st.prox6(st.sym_gradient(B, *k["w"]), 1.0 / k["alpha0"])
    sd = st.sym_divergence(y2, *k["w"])
    for comp, pos, want in k["values"]:
        assert abs(abs(ki.at(sd[comp], pos)) - want) < EPS, (comp, pos)


def test_tgv2_adapt_step(kats):
    k = kats["tgv2_adapt_step"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=None, centered=k["centered"])
    p = so.Params(sigma=k["sigma0"], tau=k["tau0"])
    e = ki.image(W, H, T)
    so.tgv2_adapt_step(p, op, e, [e, e, e], ki.b1_std(W, H, C), (1.0, 1.0, 1.0))
    assert abs(p.sigma - k["sigma"]) < EPS and abs(p.tau - k["tau"]) < EPS


def test_tgv2_norm(kats):
    k = kats["tgv2_norm"]
    W, H, T = k["dims"]
    for case in k["cases"]:
        s = complex(case["scale"]) if isinstance(case["scale"], str) else case["scale"]
        x1 = s * ki.image(W, H, T)
        x2 = [ki.image(W, H, T)] * 3
        v = st.tgv2_norm(x1, x2, k["alpha0"], k["alpha1"], *case["w"])
        assert abs(v - case["value"]) < EPS * max(1.0, 1e-3 * case["value"]), (case, v)


def test_tgv2_gstar_and_gap(kats):
    for name in ("tgv2_gstar", "tgv2_pdgap", "ictgv2_gstar"):
        k = kats[name]
        W, H, T, C, op, d, z, p = _gap_setup(k)
        x = ki.image(W, H, T)
        b1 = ki.b1_std(W, H, C)
        w = (1.0, 1.0, 1.0)
        y1 = [np.zeros_like(x) for _ in range(3)]
        y2 = [np.zeros_like(x) for _ in range(6)]
        if name == "tgv2_gstar":
            v = so.tgv2_gstar(p, op, x, y1, y2, z, d, b1, w)
        elif name == "tgv2_pdgap":
            v = so.tgv2_gap(p, op, x, [x, x, x], y1, y2, z, d, b1, w)
        else:
            v = so.ictgv2_gstar(p, op, x, y1, y2, y1, y2, z, d, b1, w, w)
        assert abs(v - k["value"]) / k["value"] < REL_GAP, (name, v)


@pytest.mark.parametrize("method", ["TGV2", "ICTGV2"])
def test_tgv2_ictgv2_iteration(kats, method):
    k = kats[method.lower() + "_iteration"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=ki.mask_of(k["mask"], W, H, T), centered=k["centered"])
    p = so.init_params(method)
    p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = k["maxIt"]
    x = so.run(method, ki.kspace(W, H, C, T), np.zeros((T, H, W), complex),
               ki.b1_std(W, H, C), op, p)
    for pos, want in k["values"]:
        assert abs(abs(ki.at(x, pos)) - want) < EPS, (pos, abs(ki.at(x, pos)), want)


# ---------------------------------------------------------------------------
# cartesian_operator.cc
# ---------------------------------------------------------------------------

def test_cartesian_forward(kats):
    k = kats["cartesian_forward"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=None, centered=k["centered"])
    img = op.forward(ki.kspace(W, H, C, T), ki.b1_std(W, H, C))
    for pos, want in k["values"]:
        assert abs(abs(ki.at(img, pos)) - want) < EPS


def test_cartesian_backward(kats):
    k = kats["cartesian_backward"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = CartesianOperator(W, H, C, T, mask=None, centered=k["centered"])
    z = op.backward(ki.image(W, H, T), ki.b1_std(W, H, C, k["b1_scales"]))
    for (x, y, c), want in k["values"]:
        assert abs(abs(z[0, c, y, x]) - want) < EPS
    for c in range(1, C):
        assert np.allclose(z[:, c], (c + 1) * z[:, 0], atol=EPS)


def test_cartesian_adjointness():
    """<K x, z> = <x, K^H z> (test_adjointness.m:1-13, cartesian_operator.cc:150-200)."""
    rng = np.random.default_rng(3)
    W, H, C, T = 12, 10, 3, 4
    for centered in (False, True):
        mask = (rng.random((T, H, W)) > 0.5).astype(float)
        op = CartesianOperator(W, H, C, T, mask=mask, centered=centered)
        x = rng.standard_normal((T, H, W)) + 1j * rng.standard_normal((T, H, W))
        z = rng.standard_normal((T, C, H, W)) + 1j * rng.standard_normal((T, C, H, W))
        b1 = rng.standard_normal((C, H, W)) + 1j * rng.standard_normal((C, H, W))
        lhs = np.vdot(op.backward(x, b1), z)
        rhs = np.vdot(x, op.forward(z.copy(), b1))
        assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_stencil_adjointness():
    """div = -grad^T and symdiv = -E^T (weighted inner product) when dx == dy."""
    rng = np.random.default_rng(5)
    T, H, W = 4, 6, 7
    w = (0.7, 0.7, 1.9)
    r = lambda: rng.standard_normal((T, H, W)) + 1j * rng.standard_normal((T, H, W))  # noqa: E731
    u = r()
    y = [r() for _ in range(3)]
    lhs = sum(np.vdot(g, c) for g, c in zip(st.gradient(u, *w), y))
    rhs = -np.vdot(u, st.divergence(y, *w))
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)
    v = [r() for _ in range(3)]
    q = [r() for _ in range(6)]
    e = st.sym_gradient(v, *w)
    lhs = sum(np.vdot(e[i], q[i]) for i in range(3)) + 2 * sum(np.vdot(e[i], q[i]) for i in range(3, 6))
    sd = st.sym_divergence(q, *w)
    rhs = -sum(np.vdot(v[i], sd[i]) for i in range(3))
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)


# ---------------------------------------------------------------------------
# coil_construction.cc
# ---------------------------------------------------------------------------

def _coil_fixture(k):
    W, H, T = k["dims"]
    C = k["coils"]
    kd = ki.kspace(W, H, C, T)
    return kd, np.ones((T, H, W)), C


def test_coil_construction_kats(kats):
    from oracle import coils as co
    k = kats["coil_construction"]
    kd, mask, C = _coil_fixture(k)
    p = co.default_params()
    u, crec = co.time_averaged_reconstruction(kd, mask)
    for (x, y), want in k["time_averaged_u_real"]:
        assert abs(u[y, x].real - want) < EPS
    for (x, y, c), want in k["time_averaged_crec_real"]:
        assert abs(crec[c, y, x].real - want) < EPS
    lap = co.laplace_periodic(np.arange(25.0).reshape(5, 5))
    for (x, y), want in k["laplace_periodic"]:
        assert abs(lap[y, x] - want) < EPS
    ua = np.abs(u).astype(complex)
    b1 = co.b1_from_u_h1(ua, crec, p)
    for (x, y, c), want in k["h1_abs_b1"]:
        assert abs(abs(b1[c, y, x]) - want) < EPS
    mi = co.find_maximum_sum(crec)
    assert mi == k["initial_index"]
    uM = co.utgv2_recon(b1[mi][None], crec[mi][None], np.zeros((5, 5), complex), [0], p)
    for (x, y), want in k["utgv2_u_real"]:
        assert abs(uM[y, x].real - want) < EPS
    x1 = co.b1_recon(b1[1] * uM, crec[1][None], 1, p["b1NrIt"], p["b1Reg"], p)[0]
    bb = b1[1] * np.exp(1j * np.angle(x1))
    for (x, y), want in k["b1recon_coil1_real"]:
        assert abs(bb[y, x].real - want) < EPS


def test_coil_construction_loop_kat(kats):
    from oracle import coils as co
    k = kats["coil_construction"]
    kd, mask, C = _coil_fixture(k)
    u, b1 = co.perform_coil_construction(kd, mask)
    for (x, y, c), want in k["loop_b1_real"]:
        assert abs(b1[c, y, x].real - want) < EPS
    for (x, y, c), want in k["loop_u_real"]:
        assert abs(u[c, y, x].real - want) < EPS


# ---------------------------------------------------------------------------
# radial operator (CUDA/test/noncartesian_operator.cc)
# ---------------------------------------------------------------------------

def test_radial_adapt_lambda_kat(kats):
    """NoncartesianOperator::AdaptLambda (noncartesian_operator.cpp:88-95) on the
    reference fixture: W / (spokesPerFrame pi / 2) k + d = 6.636."""
    from oracle import radial as rd
    from tests import kat_inputs as ki
    f, k = kats["radial_fixture"], kats["radial_adapt_lambda"]
    traj, dens, _ = ki.radial_fixture(f)
    op = rd.RadialOperator(f["width"], f["height"], f["coils"], f["frames"], traj.astype(float), dens.astype(float),
                           3.0, 8.0, 2.0)
    assert abs(op.adapt_lambda(k["k"], k["d"], f["spokesPerFrame"]) - k["value"]) < 1e-3


def test_radial_adjointness_kat(kats):
    """The reference's adjointness test (noncartesian_operator.cc:161-201) on its
    fixture with the oracle's gridding (kernel width 3, sector width 8, osf 2,
    the reference's defaults)."""
    from oracle import radial as rd
    from tests import kat_inputs as ki
    f, k = kats["radial_fixture"], kats["radial_adjointness"]
    traj, dens, b1 = ki.radial_fixture(f)
    W, H, C, T = f["width"], f["height"], f["coils"], f["frames"]
    op = rd.RadialOperator(W, H, C, T, traj.astype(float), dens.astype(float), 3.0, 8.0, 2.0)
    rng = np.random.default_rng(161)
    x = rng.random((T, C, op.S)) + 1j * rng.random((T, C, op.S))   # k-space
    y = rng.random((T, H, W)) + 1j * rng.random((T, H, W))          # image
    kx = op.forward(x.copy(), b1)    # ForwardOperation: k-space -> image
    khy = op.backward(y, b1)         # BackwardOperation: image -> k-space
    d = np.vdot(y, kx) - np.vdot(khy, x)
    assert abs(d.real) < k["tolerance"] and abs(d.imag) < k["tolerance"]
    assert abs(d) < 1e-12 * abs(np.vdot(y, kx))
