"""Properties of the oracle's TVtemp and ICTV pieces (CPU, float64).

The reference tree has no known-answer tests for these two methods; their
building blocks are pinned here by the identities the reference's
definitions imply: Divergence_temp is the negative adjoint of Gradient_temp
(utils.cpp:134-143, 795-805), ProximalMap1D projects onto the unit ball
(utils.cpp:1307-1311), ICTVNorm combines two TV norms (utils.cpp:1221-1242).
"""

import numpy as np
import pytest

from oracle import solvers as so
from oracle import stencils as st
from oracle.cartesian import CartesianOperator


def _c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_temporal_divergence_is_the_negative_adjoint_of_the_gradient():
    rng = np.random.default_rng(0)
    u, y = _c(rng, (5, 4, 3)), _c(rng, (5, 4, 3))
    for dt in (1.0, 0.37):
        lhs = np.vdot(st.gradient_temp(u, dt)[0], y)
        rhs = -np.vdot(u, st.divergence_temp([y], dt))
        assert abs(lhs - rhs) < 1e-12 * abs(lhs)
    # the temporal component of the full gradient with dx = dy = 1
    assert np.allclose(st.gradient_temp(u, 0.5)[0], st.gradient(u, 1.0, 1.0, 0.5)[2])


def test_prox1_projects_onto_the_unit_ball():
    rng = np.random.default_rng(1)
    y = [3.0 * _c(rng, (6, 5, 4))]
    p = st.prox1(y, 1.0)[0]
    assert np.all(np.abs(p) <= 1.0 + 1e-12)
    inside = np.abs(y[0]) <= 1.0
    assert np.array_equal(p[inside], y[0][inside])
    assert np.allclose(np.angle(p[~inside]), np.angle(y[0][~inside]))


def test_ictv_norm_combines_two_tv_norms():
    rng = np.random.default_rng(2)
    x1, x3 = _c(rng, (4, 6, 5)), _c(rng, (4, 6, 5))
    w1, w2 = (0.5, 0.5, 2.0), (1.5, 1.5, 0.25)
    for alpha in (0.3, 0.5, 0.8):
        m = min(alpha, 1.0 - alpha)
        ref = (alpha / m) * st.tv_norm(x1 - x3, *w1) + ((1.0 - alpha) / m) * st.tv_norm(x3, *w2)
        assert np.isclose(st.ictv_norm(x1, x3, 1.0, alpha, w1, w2), ref)
    # x3 = 0 leaves the first branch
    assert np.isclose(st.ictv_norm(x1, 0 * x1, 2.0, 0.5, w1, w2), 2.0 * st.tv_norm(x1, *w1))


@pytest.mark.filterwarnings("ignore:invalid value encountered:RuntimeWarning")  # the step rule's 0/0
def test_loops_keep_a_zero_problem_at_zero_and_follow_the_schedule():
    rng = np.random.default_rng(3)
    T, C, H, W = 3, 2, 6, 5
    mask = (rng.random((T, H, W)) > 0.5).astype(float)
    op = CartesianOperator(W, H, C, T, mask=mask, centered=False)
    b1 = _c(rng, (C, H, W))
    zero = np.zeros((T, C, H, W), complex)
    for method in ("TVTEMP", "ICTV"):
        p = so.init_params(method)
        p.maxIt, p.lam = 12, 2.0
        tr = {}
        x = so.run(method, zero, np.zeros((T, H, W), complex), b1, op, p, tr)
        assert np.all(x == 0)
        assert tr["iterations"] == 12 and len(tr["steps"]) == 12


def test_ictv_step_rule_sees_the_data_term_only():
    """ICTV::AdaptStepSize overwrites its regulariser sums (ictv.cpp:104-125):
    nKx is |K e1| whatever e3 is."""
    rng = np.random.default_rng(4)
    T, C, H, W = 2, 2, 5, 4
    op = CartesianOperator(W, H, C, T, mask=None, centered=False)
    b1 = _c(rng, (C, H, W))
    e1, e3 = _c(rng, (T, H, W)), _c(rng, (T, H, W))
    p = so.init_params("ICTV")
    nKx_a, nx_a = so.ictv_adapt_step(p.copy(), op, e1, e3, b1)
    nKx_b, nx_b = so.ictv_adapt_step(p.copy(), op, e1, 10 * e3, b1)
    assert np.isclose(nKx_a, nKx_b)
    assert np.isclose(nKx_a, np.linalg.norm(op.backward(e1, b1).ravel()))
    assert nx_b > nx_a
