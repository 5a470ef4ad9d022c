"""TV / TVtemp / TGV2 / ICTV / ICTGV2 primal-dual loops (float64), following
the reference C++.

Test infrastructure (see ``oracle/__init__``).  The loop order, the step-size
schedule (adapt at k < 10 or k % 50 == 0), the gap cadence and the early-exit
points follow ``CUDA/src/tv.cpp:99-200``, ``tv_temp.cpp:95-182``,
``tgv2.cpp:180-338``, ``ictv.cpp:202-370`` and ``ictgv2.cpp:294-492`` (the
drop-in semantics), not the MATLAB variants, which adapt every iteration.

``norm1`` of a complex vector: the reference calls AGILE ``norm1`` in the
G* terms (tv.cpp:225, tgv2.cpp:150-160, ictgv2.cpp:205-226).  Which of
sum|z| or sum(|re|+|im|) it computes is not visible in the tree; the gap
goldens of CUDA/test/tv.cc:376,435 and tgv2.cc:427,494 decide it (see
tests/test_oracle_kats.py); the default below is the one they select.
"""

import numpy as np

from . import stencils as st
from .cartesian import CartesianOperator  # noqa: F401  (re-export for callers)

NORM1_MODE = "abs"


def norm1(v, mode=None):
    mode = mode or NORM1_MODE
    if mode == "abs":
        return float(np.sum(np.abs(v)))
    return float(np.sum(np.abs(v.real)) + np.sum(np.abs(v.imag)))


def dot_re(a, b):
    """Re <a, b> (AGILE getScalarProduct, real part)."""
    return float(np.real(np.vdot(a, b)))


class Params:
    """Subset of ``PDParams``/``TGV2Params``/``ICTGV2Params``
    (pd_recon.h:34-74, tgv2.h:9-16, ictgv2.h:9-21) the loops read."""

    def __init__(self, **kw):
        self.maxIt = 500
        self.stopPDGap = 0.0
        self.sigma = 1.0 / 3.0
        self.tau = 1.0 / 3.0
        self.sigmaTauRatio = 1.0
        self.timeSpaceWeight = 5.0
        self.timeSpaceWeight2 = 2.5
        self.lam = 1.0
        self.alpha0 = np.sqrt(2.0)
        self.alpha1 = 1.0
        self.alpha = 0.6423
        self.dt = 1.0  # TVtemp only: its temporal step (no time-space weighting)
        self.debug = False
        self.debugstep = 1
        self.verbose = False
        for k, v in kw.items():
            if not hasattr(self, k):
                raise KeyError(k)
            setattr(self, k, v)

    def copy(self):
        p = Params()
        p.__dict__.update(self.__dict__)
        return p


def init_params(method):
    """The InitParams() defaults of the reference solvers (tv.cpp:39-57,
    tv_temp.cpp:39-54, tgv2.cpp:36-56, ictv.cpp:37-60, ictgv2.cpp:37-63);
    lambda is left for adapt_lambda."""
    p = Params()
    if method == "TVTEMP":
        p.dt = 1.0
        p.adapt_kd = (0.4 * 0.2991, 10.0 * 0.2991)
    elif method == "ICTV":
        p.timeSpaceWeight = 4.0
        p.timeSpaceWeight2 = 0.5
        p.alpha = 0.5
        p.adapt_kd = (0.4 / (5.1191 * 0.35), 10.0 / (5.1191 * 0.35))
    elif method == "TV":
        p.timeSpaceWeight = 5.0
        p.adapt_kd = (0.4 * 0.2991, 10.0 * 0.2991)
    elif method == "TGV2":
        p.timeSpaceWeight = 5.0
        p.adapt_kd = (0.4 * 0.2991, 10.0 * 0.2991)
    elif method == "ICTGV2":
        p.timeSpaceWeight = 6.5
        p.timeSpaceWeight2 = 2.5
        p.alpha = 0.6423
        p.adapt_kd = (0.4 / (5.1191 * 0.35), 10.0 / (5.1191 * 0.35))
    else:
        raise ValueError(method)
    return p


def _gap_due(p, k):
    return ((p.verbose and (k < 10 or k % 50 == 0))
            or (p.debug and p.debugstep > 0 and k % p.debugstep == 0)
            or (p.stopPDGap > 0 and k % 20 == 0))


def _step_due(k):
    return k < 10 or k % 50 == 0


# ---------------------------------------------------------------------------
# TV
# ---------------------------------------------------------------------------

def tv_adapt_step(p, op, e, b1, w):
    """``TV::AdaptStepSize`` (tv.cpp:79-97)."""
    g = st.gradient(e, *w)
    kz = op.backward(e, b1)
    s = sum(dot_re(c, c) for c in g) + dot_re(kz, kz)
    nKx = np.sqrt(abs(s))
    nx = np.linalg.norm(e.ravel())
    p.sigma, p.tau = st.step_rule(p.sigma, p.tau, nKx, nx, p.sigmaTauRatio)
    return nKx, nx


def tv_gstar(p, op, x, y, z, d, b1, w):
    """``TV::ComputeGStar`` (tv.cpp:202-226)."""
    r = op.backward(x, b1) - d
    g1 = 0.5 * p.lam * dot_re(r, r)
    g2 = dot_re(d, z) + dot_re(z, z) / (2.0 * p.lam)
    g3 = norm1(op.forward(z, b1) - st.divergence(y, *w))
    return g1 + g2 + g3


def tv_gap(p, op, x, y, z, d, b1, w):
    """``TV::ComputePDGap`` (tv.cpp:228-235)."""
    return abs(tv_gstar(p, op, x, y, z, d, b1, w) + st.tv_norm(x, *w))


def tv(data, x, b1, op, p, trace=None, k0=0):
    """``TV::IterativeReconstruction`` (tv.cpp:99-200).  ``x`` is the initial
    image (T,H,W); returns the final image.  ``trace`` (a dict) collects the
    gap history ("PDGap") and the (sigma, tau) sequence."""
    p = p.copy()
    ds, dt = st.time_space_weights(p.timeSpaceWeight)
    w = (ds, ds, dt)
    N = x.size
    x = x.astype(np.complex128).copy()
    ext = x.copy()
    y = [np.zeros_like(x) for _ in range(3)]
    z = np.zeros_like(data, dtype=np.complex128)
    gaps, steps = [], []
    k = k0
    while k < p.maxIt:
        g = st.gradient(ext, *w)
        y = [y[i] + p.sigma * g[i] for i in range(3)]
        z = z + p.sigma * op.backward(ext, b1)
        y = st.prox3(y, 1.0)
        z = (z - p.sigma * data) * (1.0 / (1.0 + p.sigma / p.lam))
        img = op.forward(z, b1)
        xn = x - p.tau * (img - st.divergence(y, *w))
        ext = 2.0 * xn - x
        x = xn
        if _step_due(k):
            tv_adapt_step(p, op, ext - x, b1, w)
        steps.append((p.sigma, p.tau))
        if _gap_due(p, k):
            gap = tv_gap(p, op, x, y, z, data, b1, w) / N
            gaps.append(gap)
            if gap < p.stopPDGap:
                break
        k += 1
    if trace is not None:
        trace.update(PDGap=gaps, steps=steps, iterations=k, y=y, z=z, w=w)
    return x


# ---------------------------------------------------------------------------
# TGV2
# ---------------------------------------------------------------------------

def tgv2_adapt_step(p, op, e1, e2, b1, w):
    """``TGV2::AdaptStepSize`` (tgv2.cpp:89-128)."""
    g = st.gradient(e1, *w)
    g = [g[i] - e2[i] for i in range(3)]
    s = st.sum_sq3(g) + st.sum_sq6(st.sym_gradient(e2, *w))
    kz = op.backward(e1, b1)
    tot = float(np.sum(s)) + float(np.sum(np.abs(kz) ** 2))
    nKx = np.sqrt(abs(tot))
    nx = np.sqrt(float(np.sum(np.abs(e1) ** 2 + st.sum_sq3(e2))))
    p.sigma, p.tau = st.step_rule(p.sigma, p.tau, nKx, nx, p.sigmaTauRatio)
    return nKx, nx


def tgv2_gstar(p, op, x1, y1, y2, z, d, b1, w):
    """``TGV2::ComputeGStar`` (tgv2.cpp:130-164)."""
    r = op.backward(x1, b1) - d
    g1 = 0.5 * p.lam * dot_re(r, r)
    g2 = dot_re(d, z) + dot_re(z, z) / (2.0 * p.lam)
    g3 = norm1(op.forward(z, b1) - st.divergence(y1, *w))
    sd = st.sym_divergence(y2, *w)
    g4 = sum(norm1(sd[i] + y1[i]) for i in range(3))
    return g1 + g2 + g3 + g4


def tgv2_gap(p, op, x1, x2, y1, y2, z, d, b1, w):
    """``TGV2::ComputePDGap`` (tgv2.cpp:166-176)."""
    return abs(tgv2_gstar(p, op, x1, y1, y2, z, d, b1, w)
               + st.tgv2_norm(x1, x2, p.alpha0, p.alpha1, *w))


def tgv2(data, x1, b1, op, p, trace=None, k0=0):
    """``TGV2::IterativeReconstruction`` (tgv2.cpp:180-338)."""
    p = p.copy()
    ds, dt = st.time_space_weights(p.timeSpaceWeight)
    w = (ds, ds, dt)
    N = x1.size
    x1 = x1.astype(np.complex128).copy()
    ext1 = x1.copy()
    x2 = [np.zeros_like(x1) for _ in range(3)]
    ext2 = [np.zeros_like(x1) for _ in range(3)]
    y1 = [np.zeros_like(x1) for _ in range(3)]
    y2 = [np.zeros_like(x1) for _ in range(6)]
    z = np.zeros_like(data, dtype=np.complex128)
    gaps, steps = [], []
    k = k0
    while k < p.maxIt:
        g = st.gradient(ext1, *w)
        y1 = [y1[i] + p.sigma * (g[i] - ext2[i]) for i in range(3)]
        e = st.sym_gradient(ext2, *w)
        y2 = [y2[i] + p.sigma * e[i] for i in range(6)]
        z = z + p.sigma * op.backward(ext1, b1)
        y1 = st.prox3(y1, 1.0 / p.alpha1)
        y2 = st.prox6(y2, 1.0 / p.alpha0)
        z = (z - p.sigma * data) * (1.0 / (1.0 + p.sigma / p.lam))
        img = op.forward(z, b1)
        x1n = x1 - p.tau * (img - st.divergence(y1, *w))
        sd = st.sym_divergence(y2, *w)
        x2n = [x2[i] + p.tau * (y1[i] + sd[i]) for i in range(3)]
        ext1 = 2.0 * x1n - x1
        ext2 = [2.0 * x2n[i] - x2[i] for i in range(3)]
        x1, x2 = x1n, x2n
        if _step_due(k):
            tgv2_adapt_step(p, op, ext1 - x1, [ext2[i] - x2[i] for i in range(3)], b1, w)
        steps.append((p.sigma, p.tau))
        if _gap_due(p, k):
            gap = tgv2_gap(p, op, x1, x2, y1, y2, z, data, b1, w) / N
            if gap < p.stopPDGap:
                break
            gaps.append(gap)
        k += 1
    if trace is not None:
        trace.update(PDGap=gaps, steps=steps, iterations=k, x2=x2, w=w)
    return x1


# ---------------------------------------------------------------------------
# ICTGV2
# ---------------------------------------------------------------------------

def ictgv2_weights(p):
    ds, dt = st.time_space_weights(p.timeSpaceWeight)
    ds2, dt2 = st.time_space_weights(p.timeSpaceWeight2)
    return (ds, ds, dt), (ds2, ds2, dt2)


def ictgv2_adapt_step(p, op, e1, e2, e3, e4, b1, w1, w2):
    """``ICTGV2::AdaptStepSize`` (ictgv2.cpp:97-161)."""
    g = st.gradient(e1 - e3, *w1)
    s = st.sum_sq3([g[i] - e2[i] for i in range(3)])
    s = s + st.sum_sq6(st.sym_gradient(e2, *w1))
    g = st.gradient(e3, *w2)
    s = s + st.sum_sq3([g[i] - e4[i] for i in range(3)])
    s = s + st.sum_sq6(st.sym_gradient(e4, *w2))
    kz = op.backward(e1, b1)
    tot = float(np.sum(s)) + float(np.sum(np.abs(kz) ** 2))
    nKx = np.sqrt(abs(tot))
    sx = np.abs(e1) ** 2 + st.sum_sq3(e2) + np.abs(e3) ** 2 + st.sum_sq3(e4)
    nx = np.sqrt(float(np.sum(sx)))
    p.sigma, p.tau = st.step_rule(p.sigma, p.tau, nKx, nx, p.sigmaTauRatio)
    return nKx, nx


def ictgv2_data_fidelity(p, op, x1, d, b1):
    """``ICTGV2::ComputeDataFidelity`` (ictgv2.cpp:163-176): lambda/2 times
    the (unsquared) 2-norm of K x1 - d."""
    r = op.backward(x1, b1) - d
    return float(np.linalg.norm(r.ravel())) * p.lam / 2.0


def ictgv2_gstar(p, op, x1, y1, y2, y3, y4, z, d, b1, w1, w2):
    """``ICTGV2::ComputeGStar`` (ictgv2.cpp:178-232)."""
    r = op.backward(x1, b1) - d
    g1 = 0.5 * p.lam * dot_re(r, r)
    g2 = dot_re(d, z) + dot_re(z, z) / (2.0 * p.lam)
    div1 = st.divergence(y1, *w1)
    g3 = norm1(op.forward(z, b1) - div1)
    sd = st.sym_divergence(y2, *w1)
    g4 = sum(norm1(sd[i] + y1[i]) for i in range(3))
    g5 = norm1(div1 - st.divergence(y3, *w2))
    sd = st.sym_divergence(y4, *w2)
    g6 = sum(norm1(sd[i] + y3[i]) for i in range(3))
    return g1 + g2 + g3 + g4 + g5 + g6


def ictgv2_gap(p, op, x1, x2, x3, x4, y1, y2, y3, y4, z, d, b1, w1, w2):
    """``ICTGV2::ComputePDGap`` (ictgv2.cpp:234-249)."""
    g = ictgv2_gstar(p, op, x1, y1, y2, y3, y4, z, d, b1, w1, w2)
    n = st.ictgv2_norm(x1, x2, x3, x4, p.alpha0, p.alpha1, p.alpha, w1, w2)
    return abs(g + n)


def ictgv2(data, x1, b1, op, p, trace=None, k0=0):
    """``ICTGV2::IterativeReconstruction`` (ictgv2.cpp:294-492)."""
    p = p.copy()
    w1, w2 = ictgv2_weights(p)
    N = x1.size
    x1 = x1.astype(np.complex128).copy()
    ext1 = x1.copy()
    zero = lambda n: [np.zeros_like(x1) for _ in range(n)]  # noqa: E731
    x3, ext3 = np.zeros_like(x1), np.zeros_like(x1)
    x2, ext2, x4, ext4 = zero(3), zero(3), zero(3), zero(3)
    y1, y3, y2, y4 = zero(3), zero(3), zero(6), zero(6)
    z = np.zeros_like(data, dtype=np.complex128)
    m = min(p.alpha, 1.0 - p.alpha)
    fid = [ictgv2_data_fidelity(p, op, x1, data, b1)]
    nrm = [st.ictgv2_norm(x1, x2, x3, x4, p.alpha0, p.alpha1, p.alpha, w1, w2)]
    gaps, steps = [], []
    k = k0
    while k < p.maxIt:
        g = st.gradient(ext1 - ext3, *w1)
        y1 = [y1[i] + p.sigma * (g[i] - ext2[i]) for i in range(3)]
        g = st.gradient(ext3, *w2)
        y3 = [y3[i] + p.sigma * (g[i] - ext4[i]) for i in range(3)]
        e = st.sym_gradient(ext2, *w1)
        y2 = [y2[i] + p.sigma * e[i] for i in range(6)]
        e = st.sym_gradient(ext4, *w2)
        y4 = [y4[i] + p.sigma * e[i] for i in range(6)]
        z = z + p.sigma * op.backward(ext1, b1)
        y1 = st.prox3(y1, 1.0 / (p.alpha1 * (p.alpha / m)))
        y2 = st.prox6(y2, 1.0 / (p.alpha0 * (p.alpha / m)))
        y3 = st.prox3(y3, 1.0 / (p.alpha1 * ((1.0 - p.alpha) / m)))
        y4 = st.prox6(y4, 1.0 / (p.alpha0 * ((1.0 - p.alpha) / m)))
        z = (z - p.sigma * data) * (1.0 / (1.0 + p.sigma / p.lam))
        img = op.forward(z, b1)
        div1 = st.divergence(y1, *w1)
        x1n = x1 - p.tau * (img - div1)
        sd = st.sym_divergence(y2, *w1)
        x2n = [x2[i] + p.tau * (y1[i] + sd[i]) for i in range(3)]
        div3 = st.divergence(y3, *w2)
        x3n = x3 - p.tau * (div1 - div3)
        sd = st.sym_divergence(y4, *w2)
        x4n = [x4[i] + p.tau * (y3[i] + sd[i]) for i in range(3)]
        ext1 = 2.0 * x1n - x1
        ext3 = 2.0 * x3n - x3
        ext2 = [2.0 * x2n[i] - x2[i] for i in range(3)]
        ext4 = [2.0 * x4n[i] - x4[i] for i in range(3)]
        x1, x2, x3, x4 = x1n, x2n, x3n, x4n
        if _step_due(k):
            ictgv2_adapt_step(p, op, ext1 - x1, [ext2[i] - x2[i] for i in range(3)],
                              ext3 - x3, [ext4[i] - x4[i] for i in range(3)], b1, w1, w2)
        steps.append((p.sigma, p.tau))
        if _gap_due(p, k):
            gap = ictgv2_gap(p, op, x1, x2, x3, x4, y1, y2, y3, y4, z, data, b1, w1, w2) / N
            gaps.append(gap)
            nrm.append(st.ictgv2_norm(x1, x2, x3, x4, p.alpha0, p.alpha1, p.alpha, w1, w2))
            fid.append(ictgv2_data_fidelity(p, op, x1, data, b1))
            if gap < p.stopPDGap:
                break
        k += 1
    if trace is not None:
        trace.update(PDGap=gaps, ICTGVnorm=nrm, DATAfidelity=fid, steps=steps,
                     iterations=k, x3=x3, w1=w1, w2=w2)
    return x1


# ---------------------------------------------------------------------------
# TVtemp
# ---------------------------------------------------------------------------

def tvtemp_adapt_step(p, op, e, b1):
    """``TVTEMP::AdaptStepSize`` (tv_temp.cpp:80-95)."""
    g = st.gradient_temp(e, p.dt)
    kz = op.backward(e, b1)
    nKx = np.sqrt(abs(dot_re(g[0], g[0]) + dot_re(kz, kz)))
    nx = np.linalg.norm(e.ravel())
    p.sigma, p.tau = st.step_rule(p.sigma, p.tau, nKx, nx, p.sigmaTauRatio)
    return nKx, nx


def tvtemp_gap(p, op, x, y, z, d, b1):
    """``TVTEMP::ComputeGStar`` / ``ComputePDGap`` (tv_temp.cpp:184-224): the
    regulariser term is the full TVNorm with dx = dy = 1 and the run's dt."""
    r = op.backward(x, b1) - d
    g1 = 0.5 * p.lam * dot_re(r, r)
    g2 = dot_re(d, z) + dot_re(z, z) / (2.0 * p.lam)
    g3 = norm1(op.forward(z, b1) - st.divergence_temp(y, p.dt))
    return abs(g1 + g2 + g3 + st.tv_norm(x, 1.0, 1.0, p.dt))


def tvtemp(data, x, b1, op, p, trace=None, k0=0):
    """``TVTEMP::IterativeReconstruction`` (tv_temp.cpp:95-182): TV along t
    only, no time-space weighting."""
    p = p.copy()
    N = x.size
    x = x.astype(np.complex128).copy()
    ext = x.copy()
    y = [np.zeros_like(x)]
    z = np.zeros_like(data, dtype=np.complex128)
    gaps, steps = [], []
    k = k0
    while k < p.maxIt:
        g = st.gradient_temp(ext, p.dt)
        y = [y[0] + p.sigma * g[0]]
        z = z + p.sigma * op.backward(ext, b1)
        y = st.prox1(y, 1.0)
        z = (z - p.sigma * data) * (1.0 / (1.0 + p.sigma / p.lam))
        img = op.forward(z, b1)
        xn = x - p.tau * (img - st.divergence_temp(y, p.dt))
        ext = 2.0 * xn - x
        x = xn
        if _step_due(k):
            tvtemp_adapt_step(p, op, ext - x, b1)
        steps.append((p.sigma, p.tau))
        if _gap_due(p, k):
            gap = tvtemp_gap(p, op, x, y, z, data, b1) / N
            gaps.append(gap)
            if gap < p.stopPDGap:
                break
        k += 1
    if trace is not None:
        trace.update(PDGap=gaps, steps=steps, iterations=k, y=y, z=z)
    return x


# ---------------------------------------------------------------------------
# ICTV
# ---------------------------------------------------------------------------

def ictv_adapt_step(p, op, e1, e3, b1):
    """``ICTV::AdaptStepSize`` (ictv.cpp:97-128).  The reference sums the
    gradient terms into a buffer that it overwrites before use, so only the
    data term enters nKx."""
    kz = op.backward(e1, b1)
    nKx = np.sqrt(abs(float(np.sum(np.abs(kz) ** 2))))
    nx = np.sqrt(abs(float(np.sum(np.abs(e1) ** 2 + np.abs(e3) ** 2))))
    p.sigma, p.tau = st.step_rule(p.sigma, p.tau, nKx, nx, p.sigmaTauRatio)
    return nKx, nx


def ictv_gap(p, op, x1, x3, y1, y3, z, d, b1, w1, w2):
    """``ICTV::ComputeGStar`` / ``ComputePDGap`` (ictv.cpp:146-200)."""
    r = op.backward(x1, b1) - d
    g1 = 0.5 * p.lam * dot_re(r, r)
    g2 = dot_re(d, z) + dot_re(z, z) / (2.0 * p.lam)
    div1 = st.divergence(y1, *w1)
    g3 = norm1(op.forward(z, b1) - div1)
    g5 = norm1(div1 - st.divergence(y3, *w2))
    return abs(g1 + g2 + g3 + g5 + st.ictv_norm(x1, x3, p.alpha1, p.alpha, w1, w2))


def ictv(data, x1, b1, op, p, trace=None, k0=0):
    """``ICTV::IterativeReconstruction`` (ictv.cpp:202-370): infimal
    convolution of two TV functionals with their own time-space weights."""
    p = p.copy()
    w1, w2 = ictgv2_weights(p)
    N = x1.size
    x1 = x1.astype(np.complex128).copy()
    ext1 = x1.copy()
    x3, ext3 = np.zeros_like(x1), np.zeros_like(x1)
    y1 = [np.zeros_like(x1) for _ in range(3)]
    y3 = [np.zeros_like(x1) for _ in range(3)]
    z = np.zeros_like(data, dtype=np.complex128)
    m = min(p.alpha, 1.0 - p.alpha)
    gaps, nrm, fid, steps = [], [], [], []
    k = k0
    while k < p.maxIt:
        g = st.gradient(ext1 - ext3, *w1)
        y1 = [y1[i] + p.sigma * g[i] for i in range(3)]
        g = st.gradient(ext3, *w2)
        y3 = [y3[i] + p.sigma * g[i] for i in range(3)]
        z = z + p.sigma * op.backward(ext1, b1)
        y1 = st.prox3(y1, 1.0 / (p.alpha1 * (p.alpha / m)))
        y3 = st.prox3(y3, 1.0 / (p.alpha1 * ((1.0 - p.alpha) / m)))
        z = (z - p.sigma * data) * (1.0 / (1.0 + p.sigma / p.lam))
        img = op.forward(z, b1)
        div1 = st.divergence(y1, *w1)
        x1n = x1 - p.tau * (img - div1)
        x3n = x3 - p.tau * (div1 - st.divergence(y3, *w2))
        ext1 = 2.0 * x1n - x1
        ext3 = 2.0 * x3n - x3
        x1, x3 = x1n, x3n
        if _step_due(k):
            ictv_adapt_step(p, op, ext1 - x1, ext3 - x3, b1)
        steps.append((p.sigma, p.tau))
        if _gap_due(p, k):
            gap = ictv_gap(p, op, x1, x3, y1, y3, z, data, b1, w1, w2) / N
            gaps.append(gap)
            nrm.append(st.ictv_norm(x1, x3, p.alpha1, p.alpha, w1, w2))
            fid.append(ictgv2_data_fidelity(p, op, x1, data, b1))
            if gap < p.stopPDGap:
                break
        k += 1
    if trace is not None:
        trace.update(PDGap=gaps, ictvnorm=nrm, DATAfidelity=fid, steps=steps, iterations=k, x3=x3, w1=w1, w2=w2)
    return x1


def run(method, data, x0, b1, op, p, trace=None, k0=0):
    """Runs ``method``'s loop with the iteration counter starting at k0 (the
    step rule and the gap cadence read the counter; k0 > 0 runs iterations
    k0 .. maxIt-1, which is how the CPU timings skip the step-rule start)."""
    return {"TV": tv, "TVTEMP": tvtemp, "TGV2": tgv2, "ICTV": ictv, "ICTGV2": ictgv2}[method.upper()](
        data, x0, b1, op, p, trace, k0)
