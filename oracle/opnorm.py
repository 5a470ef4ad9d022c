"""Power-iteration operator-norm estimate in float64.

Test infrastructure (see ``oracle/__init__``): the checker of the device
estimate ``avx_operator_opnorm`` / ``avx_solver_opnorm``.

``getopnorm`` restates ``matlab/getopnorm.m:1-17``: starting from x0,
``y = K^H K x0``; then ``iters`` times ``x = y / ||y||`` (``y`` itself when
``||y|| = 0``), ``y = K^H K x``, ``l = y^H x``; the estimate of ``||K||^2`` is
``|l|``.  ``matlab/ls_pd.m:43-56`` calls it on the encoding operator
(``backward_opt`` / ``forward_opt``, here ``op.backward`` / ``op.forward``).

``method_operator`` gives K and K^H of a solver's whole primal-dual operator:
K is the linear map of the dual update and K^H the map of the primal update of
the loops in ``oracle/solvers.py`` (``tv.cpp:137-198``, ``tv_temp.cpp:94-182``,
``tgv2.cpp:234-335``, ``ictv.cpp:227-370``, ``ictgv2.cpp:334-490``).  Its dual
inner product counts the off-diagonal entries of the symmetrised gradient
twice, as ``utils.cpp`` SumOfSquares6 does in the step rule; ``dual_dot``
is that inner product.  Primal vectors are lists of components in the
solver's order (TV, TVtemp: [u]; ICTV: [u, w]; TGV2: [u, v0, v1, v2];
ICTGV2: [u, v0, v1, v2, w, s0, s1, s2]).  The test that K^H is the adjoint
of K under these inner products is ``tests/test_opnorm.py``.
"""

import numpy as np

from . import stencils as st


def getopnorm(normal, x0, iters=10, history=None):
    """``getopnorm(K, Kh, imgdims)`` with ``normal = Kh o K`` on lists of
    arrays and the start vector given (the reference draws randn).  Returns
    |l|; ``history`` (a list) receives |y^H x| after each application,
    the first against x0."""
    x = [np.asarray(c, dtype=np.complex128) for c in x0]
    y = normal(x)
    if history is not None:
        history.append(abs(sum(np.vdot(a, b) for a, b in zip(y, x))))
    lval = None
    for _ in range(iters):
        n = np.sqrt(sum(float(np.vdot(c, c).real) for c in y))
        x = [c / n for c in y] if n != 0 else y
        y = normal(x)
        lval = sum(np.vdot(a, b) for a, b in zip(y, x))  # y(:)' * x(:)
        if history is not None:
            history.append(abs(lval))
    if lval is None:
        raise ValueError("the power iteration needs at least one iteration")
    return abs(lval)


def encoding_normal(op, b1):
    """K^H K of the encoding operator on [image]."""
    return lambda xs: [op.forward(op.backward(xs[0], b1), b1)]


def _weights(method, p):
    ds, dt = st.time_space_weights(p.timeSpaceWeight)
    w1 = (ds, ds, dt)
    if method in ("ICTV", "ICTGV2"):
        ds2, dt2 = st.time_space_weights(p.timeSpaceWeight2)
        return w1, (ds2, ds2, dt2)
    return w1, None


def method_operator(method, op, b1, p):
    """(K, K^H, P) of ``method``: K maps primal components to (dual
    components, k-space), K^H maps them back."""
    method = method.upper()
    w1, w2 = _weights(method, p)
    A = lambda u: op.backward(u, b1)  # noqa: E731
    Ah = lambda z: op.forward(z, b1)  # noqa: E731

    if method == "TV":
        def K(x):
            return st.gradient(x[0], *w1), A(x[0])

        def Kh(d, z):
            return [Ah(z) - st.divergence(d, *w1)]
        return K, Kh, 1
    if method == "TVTEMP":
        def K(x):
            return st.gradient_temp(x[0], p.dt), A(x[0])

        def Kh(d, z):
            return [Ah(z) - st.divergence_temp(d, p.dt)]
        return K, Kh, 1
    if method == "ICTV":
        def K(x):
            return st.gradient(x[0] - x[1], *w1) + st.gradient(x[1], *w2), A(x[0])

        def Kh(d, z):
            div1 = st.divergence(d[0:3], *w1)
            return [Ah(z) - div1, div1 - st.divergence(d[3:6], *w2)]
        return K, Kh, 2
    if method in ("TGV2", "ICTGV2"):
        def branch(u, v, w):
            g = st.gradient(u, *w)
            return [g[i] - v[i] for i in range(3)] + st.sym_gradient(v, *w)

        def branch_h(d, w):
            sd = st.sym_divergence(d[3:9], *w)
            return st.divergence(d[0:3], *w), [-(d[i] + sd[i]) for i in range(3)]

        if method == "TGV2":
            def K(x):
                return branch(x[0], x[1:4], w1), A(x[0])

            def Kh(d, z):
                div1, v = branch_h(d, w1)
                return [Ah(z) - div1] + v
            return K, Kh, 4

        def K(x):
            return branch(x[0] - x[4], x[1:4], w1) + branch(x[4], x[5:8], w2), A(x[0])

        def Kh(d, z):
            div1, v = branch_h(d[0:9], w1)
            div3, s = branch_h(d[9:18], w2)
            return [Ah(z) - div1] + v + [div1 - div3] + s
        return K, Kh, 8
    raise ValueError(method)


def dual_dot(method, a, b):
    """Dual inner product sum conj(a) b, with the symmetrised gradient's
    off-diagonal components (3..5 of every 9-component branch) counted twice."""
    method = method.upper()
    tot = 0j
    for i, (u, v) in enumerate(zip(a, b)):
        wgt = 2.0 if method in ("TGV2", "ICTGV2") and (i % 9) >= 6 else 1.0
        tot += wgt * np.vdot(u, v)
    return tot


def method_normal(method, op, b1, p):
    K, Kh, _ = method_operator(method, op, b1, p)

    def normal(x):
        d, z = K(x)
        return Kh(d, z)
    return normal


def method_start(method, x0):
    """The start vector of the solver estimate: x0 for the image, zeros for
    the auxiliary components."""
    _P = {"TV": 1, "TVTEMP": 1, "ICTV": 2, "TGV2": 4, "ICTGV2": 8}[method.upper()]
    x0 = np.asarray(x0, dtype=np.complex128)
    return [x0] + [np.zeros_like(x0) for _ in range(_P - 1)]


def opnorm_steps(l, ratio):
    """sig = s r, tau = s / r with s = 1 / sqrt(l) (tgv2_dmri.m:96-99 with
    1/||K|| in place of 1/3)."""
    L = np.sqrt(l)
    return ratio / L, 1.0 / (ratio * L)
