"""Finite differences, gradients, divergences, norms and proximal maps (float64).

Test infrastructure (see ``oracle/__init__``).  Restates the arithmetic of
``CUDA/src/utils.cpp`` of the reference on numpy arrays of shape (T, H, W).

Axis convention of the reference's AGILE ``diff3``/``bdiff3`` kernels:
dimension 1 = x (array axis 2, stride 1), dimension 2 = y (axis 1, stride W),
dimension 3 = t (axis 0, stride W*H).  Boundary semantics are pinned by
``CUDA/test/derivatives.cc:169-650``:

* forward difference D+ (``diff3``, no wrap): (D+u)_i = u_{i+1} - u_i, and 0
  at the last index;
* backward difference D- (``bdiff3``, no wrap) = -(D+)^T:  (D-u)_0 = u_0,
  (D-u)_i = u_i - u_{i-1}, (D-u)_{n-1} = -u_{n-2};
* ``diff3trans`` = (D+)^T, ``bdiff3trans`` = (D-)^T = -D+;
* wrap=True (periodic) variants, used only by the H1 coil estimation CG.
"""

import numpy as np

_AXIS = {1: 2, 2: 1, 3: 0}


def _shift(u, axis, k):
    return np.roll(u, k, axis=axis)


def diff(u, dim, wrap=False):
    """D+ along ``dim`` (AGILE ``lowlevel::diff3``; derivatives.cc:169-204)."""
    a = _AXIS[dim]
    out = _shift(u, a, -1) - u
    if not wrap:
        idx = [slice(None)] * u.ndim
        idx[a] = -1
        out[tuple(idx)] = 0
    return out


def diff_t(u, dim, wrap=False):
    """(D+)^T along ``dim`` (``diff3trans``; derivatives.cc:206-244)."""
    a = _AXIS[dim]
    if wrap:
        return _shift(u, a, 1) - u
    n = u.shape[a]
    out = np.zeros_like(u)
    src = [slice(None)] * u.ndim
    dst = [slice(None)] * u.ndim
    # + u_{j-1} for j >= 1
    src[a] = slice(0, n - 1)
    dst[a] = slice(1, n)
    out[tuple(dst)] += u[tuple(src)]
    # - u_j for j <= n-2
    src[a] = slice(0, n - 1)
    out[tuple(src)] -= u[tuple(src)]
    return out


def bdiff(u, dim, wrap=False):
    """D- along ``dim`` (``bdiff3``; derivatives.cc:246-279)."""
    a = _AXIS[dim]
    if wrap:
        return u - _shift(u, a, 1)
    return -diff_t(u, dim, wrap=False)


def bdiff_t(u, dim, wrap=False):
    """(D-)^T along ``dim`` (``bdiff3trans``; derivatives.cc:281-316)."""
    a = _AXIS[dim]
    if wrap:
        return u - _shift(u, a, -1)
    return -diff(u, dim, wrap=False)


# ---------------------------------------------------------------------------
# vector operators (utils.cpp)
# ---------------------------------------------------------------------------

def gradient(u, dx=1.0, dy=1.0, dt=1.0):
    """``utils::Gradient`` (utils.cpp:99-118): (D+x u/dx, D+y u/dy, D+t u/dt)."""
    return [diff(u, 1) / dx, diff(u, 2) / dy, diff(u, 3) / dt]


def divergence(y, dx=1.0, dy=1.0, dt=1.0):
    """``utils::Divergence`` (utils.cpp:733-757) = -(grad)^T y."""
    return -(diff_t(y[0], 1) / dx + diff_t(y[1], 2) / dy + diff_t(y[2], 3) / dt)


def gradient_temp(u, dt=1.0):
    """``utils::Gradient_temp`` (utils.cpp:134-143): [D+t u / dt]."""
    return [diff(u, 3) / dt]


def divergence_temp(y, dt=1.0):
    """``utils::Divergence_temp`` (utils.cpp:795-805) = -(D+t)^T y / dt."""
    return -(diff_t(y[0], 3) / dt)


def prox1(y, scale):
    """``utils::ProximalMap1D`` (utils.cpp:1307-1311): y / max(1, scale*|y|)."""
    d = np.maximum(1.0, scale * np.abs(y[0]))
    return [y[0] / d]


def ictv_norm(x1, x3, alpha1, alpha, w1, w2):
    """``utils::ICTVNorm`` (utils.cpp:1221-1242)."""
    m = min(alpha, 1.0 - alpha)
    return (alpha1 * (alpha / m) * tv_norm(x1 - x3, *w1)
            + alpha1 * ((1.0 - alpha) / m) * tv_norm(x3, *w2))


def sym_gradient(v, dx=1.0, dy=1.0, dt=1.0):
    """``utils::SymmetricGradient`` 7-argument form used by the PD loops
    (utils.cpp:397-456).  Off-diagonal order (xy, xt, yt).  The yt term
    divides its y-difference by ``dx`` (utils.cpp:453), as the reference does."""
    e0 = bdiff(v[0], 1) / dx
    e1 = bdiff(v[1], 2) / dy
    e2 = bdiff(v[2], 3) / dt
    e3 = bdiff(v[0], 2) / (2.0 * dy) + bdiff(v[1], 1) / (2.0 * dx)
    e4 = bdiff(v[0], 3) / (2.0 * dt) + bdiff(v[2], 1) / (2.0 * dx)
    e5 = bdiff(v[1], 3) / (2.0 * dt) + bdiff(v[2], 2) / (2.0 * dx)
    return [e0, e1, e2, e3, e4, e5]


def sym_divergence(w, dx=1.0, dy=1.0, dt=1.0):
    """``utils::SymmetricDivergence`` 8-argument form (utils.cpp:961-1012)."""
    d0 = -(bdiff_t(w[0], 1) / dx + bdiff_t(w[3], 2) / dy + bdiff_t(w[4], 3) / dt)
    d1 = -(bdiff_t(w[3], 1) / dx + bdiff_t(w[1], 2) / dy + bdiff_t(w[5], 3) / dt)
    d2 = -(bdiff_t(w[4], 1) / dx + bdiff_t(w[5], 2) / dy + bdiff_t(w[2], 3) / dt)
    return [d0, d1, d2]


def norm3(g):
    """``utils::GradientNorm`` (utils.cpp:209-222): sqrt(sum |g_i|^2)."""
    return np.sqrt(sum(np.abs(c) ** 2 for c in g))


def norm6(g):
    """``utils::SymmetricGradientNorm`` (utils.cpp:610-631): diagonal terms
    once, off-diagonal terms twice."""
    s = np.abs(g[0]) ** 2 + np.abs(g[1]) ** 2 + np.abs(g[2]) ** 2
    s = s + 2.0 * (np.abs(g[3]) ** 2 + np.abs(g[4]) ** 2 + np.abs(g[5]) ** 2)
    return np.sqrt(s)


def prox3(y, scale):
    """``utils::ProximalMap3`` (utils.cpp:1341-1345 via
    DivideVectorScaledElementwise :1297-1305): y / max(1, scale*|y|_3)."""
    d = np.maximum(1.0, scale * norm3(y))
    return [c / d for c in y]


def prox6(y, scale):
    """``utils::ProximalMap6`` (utils.cpp:1347-1351)."""
    d = np.maximum(1.0, scale * norm6(y))
    return [c / d for c in y]


def sum_sq3(x):
    """``utils::SumOfSquares3`` (utils.cpp:1398-1406)."""
    return sum(np.abs(c) ** 2 for c in x)


def sum_sq6(x):
    """``utils::SumOfSquares6`` (utils.cpp:1408-1418)."""
    return (np.abs(x[0]) ** 2 + np.abs(x[1]) ** 2 + np.abs(x[2]) ** 2
            + 2.0 * (np.abs(x[3]) ** 2 + np.abs(x[4]) ** 2 + np.abs(x[5]) ** 2))


def tv_norm(u, dx=1.0, dy=1.0, dt=1.0):
    """``utils::TVNorm`` (utils.cpp:1119-1132): sum_p |grad u|_3."""
    return float(np.sum(norm3(gradient(u, dx, dy, dt))))


def tgv2_norm(x1, x2, alpha0, alpha1, dx=1.0, dy=1.0, dt=1.0):
    """``utils::TGV2Norm`` (utils.cpp:1179-1197)."""
    g = gradient(x1, dx, dy, dt)
    g = [g[i] - x2[i] for i in range(3)]
    e = sym_gradient(x2, dx, dy, dt)
    return float(alpha1 * np.sum(norm3(g)) + alpha0 * np.sum(norm6(e)))


def ictgv2_norm(x1, x2, x3, x4, alpha0, alpha1, alpha, w1, w2):
    """``utils::ICTGV2Norm`` (utils.cpp:1245-1287).  ``w1``/``w2`` are the
    (dx, dy, dt) triples of the two TGV branches."""
    m = min(alpha, 1.0 - alpha)
    n1 = tgv2_norm(x1 - x3, x2, alpha0, alpha1, *w1)
    n2 = tgv2_norm(x3, x4, alpha0, alpha1, *w2)
    return (alpha / m) * n1 + ((1.0 - alpha) / m) * n2


# ---------------------------------------------------------------------------
# scalar helpers
# ---------------------------------------------------------------------------

def ellipke(m, tol=1e-7):
    """Complete elliptic integral of the second kind E(m) by the
    arithmetic-geometric mean, as ``utils::Ellipke`` (utils.cpp:18-47;
    Abramowitz & Stegun 17.6).  Pinned by CUDA/test/utils.cc:6-12."""
    if m < 0 or m > 1:
        raise ValueError("Ellipke: only values in [0,1] are allowed")
    a0, b0, s0 = 1.0, np.sqrt(1.0 - m), m
    i1, mm = 0, 1.0
    a1 = a0
    while mm > tol:
        a1 = (a0 + b0) / 2.0
        b1 = np.sqrt(a0 * b0)
        c1 = (a0 - b0) / 2.0
        i1 += 1
        w1 = 2.0 ** i1 * c1 * c1
        mm = w1
        s0 += w1
        a0, b0 = a1, b1
    k = np.pi / (2.0 * a1)
    return k * (1.0 - s0 / 2.0)


def time_space_weights(tsw):
    """``PDRecon::ComputeTimeSpaceWeights`` (pd_recon.cpp:72-98).
    Returns (ds, dt) = (1/w1, 1/w2)."""
    r = 1.0 / tsw
    if 0.0 < r <= 1.0:
        e = ellipke(1.0 - r * r)
        w2 = np.pi / (2.0 * e)
        w1 = r * w2
    elif r > 1.0:
        r = 1.0 / r
        e = ellipke(1.0 - r * r)
        w1 = np.pi / (2.0 * e)
        w2 = r * w1
    else:
        raise ValueError("ComputeTimeSpaceWeights: invalid ratio")
    return 1.0 / w1, 1.0 / w2


def step_rule(sigma, tau, nKx, nx, ratio, theta=0.95):
    """``PDRecon::AdaptStepSize`` (pd_recon.cpp:40-61)."""
    tmp = nx / nKx
    if sigma * tau > tmp * tmp:
        if theta * theta * sigma * tau < tmp * tmp:
            sigma *= theta
            tau *= theta
        else:
            sigma = tmp * ratio
            tau = tmp / ratio
    return sigma, tau
