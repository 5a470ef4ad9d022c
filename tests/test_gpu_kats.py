"""The reference's own known-answer tests, run on the GPU through the C ABI.

Same expected values as tests/test_oracle_kats.py (reference_kats.json), but
every number here comes out of libavionic_core.so on the device.
"""

import numpy as np
import pytest

from tests import kat_inputs as ki

pytestmark = pytest.mark.gpu
EPS = 1e-3
REL_GAP = 2e-6


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def dev(a):
    import avionic_b200
    return avionic_b200.to_device(a)


def host(t):
    return t.cpu().numpy()


def _lin3(cols, rows, slices):
    return np.arange(cols * rows * slices, dtype=np.float64).reshape(slices, rows, cols).astype(np.complex64)


@pytest.mark.parametrize("cols,rows,slices", [(5, 5, 3), (4, 4, 3), (7, 5, 3), (5, 7, 3)])
def test_derivative_kats_match_oracle_exactly(av, cols, rows, slices):
    """derivatives.cc: the stencils are integer-exact on the linear index, so
    the device gradient / divergence / symmetric pair equal the oracle exactly."""
    from oracle import stencils as st
    a = _lin3(cols, rows, slices)
    g = [host(c) for c in av.gradient(dev(a))]
    for d in range(3):
        assert np.array_equal(g[d], st.diff(a.astype(complex), d + 1).astype(np.complex64))
    y = [a, 2 * a, 3 * a]
    div = host(av.divergence([dev(c) for c in y]))
    assert np.array_equal(div, st.divergence([c.astype(complex) for c in y]).astype(np.complex64))
    e = [host(c) for c in av.sym_gradient([dev(c) for c in y])]
    ref = st.sym_gradient([c.astype(complex) for c in y])
    for k in range(6):
        assert np.array_equal(e[k], ref[k].astype(np.complex64))
    w = [a * (k + 1) for k in range(6)]
    sd = [host(c) for c in av.sym_divergence([dev(c) for c in w])]
    ref = st.sym_divergence([c.astype(complex) for c in w])
    for k in range(3):
        assert np.array_equal(sd[k], ref[k].astype(np.complex64))


def test_ellipke_and_weights(av, kats):
    for m, want in kats["ellipke"]["cases"]:
        assert abs(av.ellipke(m) - want) < EPS
    assert np.isnan(av.ellipke(1.5))
    from oracle import stencils as st
    for tsw in (0.5, 1.4, 2.5, 5.0, 6.5):
        ds, dt = av.time_space_weights(tsw)
        rds, rdt = st.time_space_weights(tsw)
        assert abs(ds - rds) < 1e-6 * rds and abs(dt - rdt) < 1e-6 * rdt


@pytest.mark.parametrize("name", ["tv_gradient_norm", "tv_scaled_gradient_norm"])
def test_tv_gradient_norm(av, kats, name):
    k = kats[name]
    W, H, T = k["dims"]
    n = host(av.norm(av.gradient(dev(ki.image(W, H, T)), *k["w"])))
    for pos, want in k["values"]:
        assert abs(ki.at(n, pos) - want) < EPS


def test_tv_divergence_of_prox(av, kats):
    k = kats["tv_divergence_of_prox"]
    W, H, T = k["dims"]
    g = av.prox(av.gradient(dev(ki.image(W, H, T))), 1.0)
    d = host(av.divergence(g))
    for pos, want in k["values"]:
        assert abs(ki.at(d, pos).real - want) < EPS


def test_tv_norm(av, kats):
    k = kats["tv_norm"]
    W, H, T = k["dims"]
    for case in k["cases"]:
        s = complex(case["scale"]) if isinstance(case["scale"], str) else case["scale"]
        v = av.tv_norm(dev(s * ki.image(W, H, T)), *case["w"])
        assert abs(v - case["value"]) < max(EPS, 2e-6 * case["value"])


@pytest.mark.parametrize("name", ["tgv2_gradient_norms", "tgv2_scaled_gradient_norms"])
def test_tgv2_norm_fields(av, kats, name):
    import torch
    k = kats[name]
    W, H, T = k["dims"]
    N = W * H * T
    A = dev(ki.image(W, H, T))
    B = [dev(ki.image(W, H, T, start=(i + 1) * N)) for i in range(3)]
    g = av.gradient(A, *k["w"])
    g = [(g[i] - B[i]).contiguous() for i in range(3)]
    n3 = host(av.norm(g))
    n6 = host(av.norm(av.sym_gradient(B, *k["w"])))
    for pos, want in k["grad"]:
        assert abs(ki.at(n3, pos) - want) < EPS
    for pos, want in k["sym"]:
        assert abs(ki.at(n6, pos) - want) < EPS
    del torch


def test_tgv2_sym_divergence_of_prox(av, kats):
    k = kats["tgv2_sym_divergence_of_prox"]
    W, H, T = k["dims"]
    N = W * H * T
    B = [dev(ki.image(W, H, T, start=(i + 1) * N)) for i in range(3)]
    y2 = av.prox(av.sym_gradient(B, *k["w"]), 1.0 / k["alpha0"])
    sd = [host(c) for c in av.sym_divergence(y2, *k["w"])]
    for comp, pos, want in k["values"]:
        assert abs(abs(ki.at(sd[comp], pos)) - want) < EPS


def test_tgv2_norm(av, kats):
    k = kats["tgv2_norm"]
    W, H, T = k["dims"]
    for case in k["cases"]:
        s = complex(case["scale"]) if isinstance(case["scale"], str) else case["scale"]
        x2 = [dev(ki.image(W, H, T)) for _ in range(3)]
        v = av.tgv2_norm(dev(s * ki.image(W, H, T)), x2, k["alpha0"], k["alpha1"], *case["w"])
        assert abs(v - case["value"]) < max(EPS, 2e-6 * case["value"])


def _op(av, k, C=None, dft=0):
    """Cartesian operator of a KAT; dft 0 is the reference's fp32 arithmetic."""
    W, H, T = k["dims"]
    C = C or k["coils"]
    m = ki.mask_of(k.get("mask"), W, H, T)
    op = av.CartesianOperator(W, H, C, T, mask=None if m is None else dev(m), centered=k["centered"])
    op.dft_mode = dft
    return op


def _tol(dft, want):
    """The reference's 1e-3 absolute (test_utils.h:11) for the fp32 form; the
    split-BF16x3 form, which agrees with fp32 to a few 1e-6 relative, may also
    differ by 1e-5 relative from the reference's fp32 values."""
    return EPS if dft == 0 else max(EPS, 1e-5 * abs(want))


DFT = [0, 1]


@pytest.mark.parametrize("dft", DFT)
def test_cartesian_forward_backward(av, kats, dft):
    k = kats["cartesian_forward"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = _op(av, k, dft=dft)
    img = host(op.forward(dev(ki.kspace(W, H, C, T)), dev(ki.b1_std(W, H, C))))
    for pos, want in k["values"]:
        assert abs(abs(ki.at(img, pos)) - want) < _tol(dft, want)
    k = kats["cartesian_backward"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = _op(av, k, dft=dft)
    z = host(op.backward(dev(ki.image(W, H, T)), dev(ki.b1_std(W, H, C, k["b1_scales"]))))
    for (x, y, c), want in k["values"]:
        assert abs(abs(z[0, c, y, x]) - want) < _tol(dft, want)


def test_adapt_lambda(av, kats):
    k = kats["tv_adapt_lambda"]
    W, H, T = k["dims"]
    op = av.CartesianOperator(W, H, k["coils"], T, mask=dev(np.ones((T, H, W))))
    assert abs(op.adapt_lambda(k["k"], k["d"]) - k["value"]) < EPS


@pytest.mark.parametrize("method,name", [("TV", "tv_adapt_step"), ("TGV2", "tgv2_adapt_step")])
def test_adapt_step(av, kats, method, name):
    k = kats[name]
    W, H, T = k["dims"]
    C = k["coils"]
    op = _op(av, k)
    s = av.Solver(method, op)
    p = s.params
    p.sigma, p.tau = k["sigma0"], k["tau0"]
    p.dx = p.dy = p.dt = 1.0
    s.params = p
    b1 = dev(ki.b1_std(W, H, C))
    if method == "TV":
        diffs = [dev(1j * ki.image(W, H, T))]
    else:
        e = ki.image(W, H, T)
        diffs = [dev(e) for _ in range(4)]
    sig, tau = s.adapt_step_size(diffs, b1)
    assert abs(sig - k["sigma"]) < EPS and abs(tau - k["tau"]) < EPS


@pytest.mark.parametrize("name,method", [("tv_gstar", "TV"), ("tv_pdgap", "TV"), ("tgv2_gstar", "TGV2"),
                                         ("tgv2_pdgap", "TGV2"), ("ictgv2_gstar", "ICTGV2")])
def test_gstar_and_gap(av, kats, name, method):
    import torch
    k = kats[name]
    W, H, T = k["dims"]
    C = k["coils"]
    op = _op(av, k)
    s = av.Solver(method, op)
    p = s.params
    p.lambda_ = k["lambda"]
    p.dx = p.dy = p.dt = 1.0
    p.dx2 = p.dy2 = p.dt2 = 1.0
    s.params = p
    x = dev(ki.image(W, H, T))
    P = av.P_OF[av.METHODS[method]]
    D = av.D_OF[av.METHODS[method]]
    xs = [x] + [x.clone() for _ in range(P - 1)]
    if method == "TGV2" and name == "tgv2_gstar":
        xs = [x] + [torch.zeros_like(x) for _ in range(P - 1)]
    ys = [torch.zeros_like(x) for _ in range(D)]
    d = dev(ki.kspace(W, H, C, T))
    z = torch.ones_like(d)
    gstar, gap = s.compute_gap(xs, ys, z, d, dev(ki.b1_std(W, H, C)))
    v = gstar if name.endswith("gstar") else gap
    assert abs(v - k["value"]) / k["value"] < REL_GAP, (name, v)


@pytest.mark.parametrize("dft", DFT)
@pytest.mark.parametrize("method", ["TV", "TGV2", "ICTGV2"])
def test_iteration_goldens(av, kats, method, dft):
    k = kats[method.lower() + "_iteration"]
    W, H, T = k["dims"]
    C = k["coils"]
    op = _op(av, k, dft=dft)
    s = av.Solver(method, op)
    x = dev(np.zeros((T, H, W), np.complex64))
    s.run(dev(ki.kspace(W, H, C, T)), x, dev(ki.b1_std(W, H, C)))
    xr = host(x)
    for pos, want in k["values"]:
        assert abs(abs(ki.at(xr, pos)) - want) < _tol(dft, want), (pos, abs(ki.at(xr, pos)), want)
    assert s.stats().iterations == k["maxIt"]


# ---------------------------------------------------------------------------
# radial operator (CUDA/test/noncartesian_operator.cc)
# ---------------------------------------------------------------------------

def _radial_op(av, kats, osf=2.0):
    f = kats["radial_fixture"]
    traj, dens, b1 = ki.radial_fixture(f)
    op = av.RadialOperator(f["width"], f["height"], f["coils"], f["frames"], dev(traj), dev(dens),
                           f["spokesPerFrame"], 3.0, 8.0, osf)
    return op, b1


def test_radial_adapt_lambda_kat(av, kats):
    """NoncartesianOperator::AdaptLambda on the reference fixture = 6.636
    (noncartesian_operator.cc:203-211)."""
    op, _ = _radial_op(av, kats)
    k = kats["radial_adapt_lambda"]
    assert abs(op.adapt_lambda(k["k"], k["d"]) - k["value"]) < EPS


@pytest.mark.parametrize("osf", [2.0, 1.5])
def test_radial_adjointness_kat(av, kats, osf):
    """The reference's adjointness test on its fixture (noncartesian_operator.cc:161-201):
    <K^H y, x> = <y, K x> within 1e-3 absolute in both parts, here also
    within 1e-5 relative."""
    f, k = kats["radial_fixture"], kats["radial_adjointness"]
    op, b1 = _radial_op(av, kats, osf)
    W, H, C, T = f["width"], f["height"], f["coils"], f["frames"]
    rng = np.random.default_rng(161)
    x = (rng.random((T, C, op.S)) + 1j * rng.random((T, C, op.S))).astype(np.complex64)
    y = (rng.random((T, H, W)) + 1j * rng.random((T, H, W))).astype(np.complex64)
    b1d = dev(b1.astype(np.complex64))
    kx = host(op.forward(dev(x), b1d)).astype(complex)
    khy = host(op.backward(dev(y), b1d)).astype(complex)
    d = np.vdot(y.astype(complex), kx) - np.vdot(khy, x.astype(complex))
    assert abs(d.real) < k["tolerance"] and abs(d.imag) < k["tolerance"]
    assert abs(d) < 1e-5 * abs(np.vdot(y.astype(complex), kx))
