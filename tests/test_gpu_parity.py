"""CUDA path vs the float64 oracle on seeded synthetic problems.

Tolerances: operator outputs 1e-5 relative L2 (FP32 arithmetic against
FP64); adjointness <Kx, z> = <x, K^H z> to 1e-5 relative; reconstructions
1e-4 relative L2 image error, the bar the method is held to.
"""

import numpy as np
import pytest

from oracle import solvers as so
from oracle.cartesian import CartesianOperator as OCart

pytestmark = pytest.mark.gpu

REL_OP = 1e-5
REL_IMG = 1e-4


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def cplx(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


CASES = [
    # W, H, C, T, mask kind, centered
    (12, 10, 3, 4, "lines", False),
    (13, 9, 2, 3, "random", True),
    (32, 24, 4, 5, "weights", False),
    (20, 20, 3, 2, None, True),
    (96, 64, 2, 3, "lines", False),
    # whole tensor-core tiles: C W a multiple of 128 and H of 16 (two stages, one stage)
    (64, 32, 2, 3, "lines", False),
    (32, 16, 4, 2, "random", True),
]


def _mask(kind, T, H, W, rng):
    if kind is None:
        return None
    if kind == "lines":
        m = np.zeros((T, H, W), np.float32)
        for t in range(T):
            m[t, rng.choice(H, size=max(1, H // 3), replace=False), :] = 1
        return m
    if kind == "random":
        return (rng.random((T, H, W)) > 0.6).astype(np.float32)
    m = np.zeros((T, H, W), np.float32)
    for t in range(T):
        m[t, rng.choice(H, size=max(1, H // 2), replace=False), :] = 1
    return m * rng.uniform(0.3, 1.7, size=(T, H, W)).astype(np.float32)


DFT_MODES = [0, 1]  # DFT_FP32, DFT_SPLIT_BF16X3


@pytest.mark.parametrize("dft", DFT_MODES)
@pytest.mark.parametrize("W,H,C,T,kind,centered", CASES)
def test_operator_matches_oracle(av, W, H, C, T, kind, centered, dft):
    rng = np.random.default_rng(W * 1000 + H)
    mask = _mask(kind, T, H, W, rng)
    x, b1, k = cplx(rng, (T, H, W)), cplx(rng, (C, H, W)), cplx(rng, (T, C, H, W))
    op = av.CartesianOperator(W, H, C, T, mask=None if mask is None else av.to_device(mask), centered=centered)
    op.dft_mode = dft
    assert op.dft_mode == dft
    oop = OCart(W, H, C, T, mask=mask, centered=centered)
    kg = op.backward(av.to_device(x), av.to_device(b1)).cpu().numpy()
    ko = oop.backward(x.astype(complex), b1.astype(complex))
    assert rel(kg, ko) < REL_OP
    kd = av.to_device(k)
    ig = op.forward(kd, av.to_device(b1)).cpu().numpy()
    kref = k.astype(complex)
    io = oop.forward(kref, b1.astype(complex))
    assert rel(ig, io) < REL_OP
    # the input is masked in place, as in the reference
    assert rel(kd.cpu().numpy(), kref) < 1e-6 or np.linalg.norm(kref) == 0


@pytest.mark.parametrize("dft", DFT_MODES)
@pytest.mark.parametrize("W,H,C,T,kind,centered", CASES)
def test_operator_adjointness(av, W, H, C, T, kind, centered, dft):
    """test_adjointness.m:1-13 / cartesian_operator.cc:150-200 on the device."""
    rng = np.random.default_rng(7 + W)
    mask = _mask(kind, T, H, W, rng)
    if mask is not None:
        mask = (mask != 0).astype(np.float32)  # K^H is the adjoint for a 0/1 mask
    x, b1, z = cplx(rng, (T, H, W)), cplx(rng, (C, H, W)), cplx(rng, (T, C, H, W))
    op = av.CartesianOperator(W, H, C, T, mask=None if mask is None else av.to_device(mask), centered=centered)
    op.dft_mode = dft
    kx = op.backward(av.to_device(x), av.to_device(b1)).cpu().numpy().astype(complex)
    khz = op.forward(av.to_device(z), av.to_device(b1)).cpu().numpy().astype(complex)
    lhs = np.vdot(kx, z.astype(complex))
    rhs = np.vdot(x.astype(complex), khz)
    assert abs(lhs - rhs) / abs(lhs) < REL_OP


def _oracle_run(method, prob, iters, debugstep=0, stop=0.0, centered=False, u0=None):
    T, C, H, W = prob["kdata"].shape
    op = OCart(W, H, C, T, mask=prob["mask"], centered=centered)
    p = so.init_params(method)
    p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = iters
    p.debug = debugstep > 0
    p.debugstep = max(debugstep, 1)
    p.stopPDGap = stop
    x0 = np.zeros((T, H, W), complex) if u0 is None else np.repeat(u0[None].astype(complex), T, axis=0)
    tr = {}
    x = so.run(method, prob["kdata"].astype(complex), x0, prob["b1"].astype(complex), op, p, tr)
    return x, tr, p


def _gpu_run(av, method, prob, iters, debugstep=0, stop=0.0, centered=False, u0=None, dft=None):
    import torch
    T, C, H, W = prob["kdata"].shape
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=centered)
    if dft is not None:
        op.dft_mode = dft
    s = av.Solver(method, op)
    p = s.params
    p.maxIt = iters
    p.stopPDGap = stop
    s.params = p
    s.set_debug(debugstep > 0, max(debugstep, 1))
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda") if u0 is None else \
        av.to_device(np.repeat(u0[None], T, axis=0))
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))
    return x.cpu().numpy(), s


@pytest.mark.parametrize("dft", DFT_MODES)
@pytest.mark.parametrize("method", ["TV", "TVTEMP", "TGV2", "ICTV", "ICTGV2"])
@pytest.mark.parametrize("binary", [True, False])
def test_solver_matches_oracle_small(av, method, binary, dft):
    from avionic_b200 import synth
    prob = synth.small(11, binary=binary)
    xo, tro, _ = _oracle_run(method, prob, 120, debugstep=10)
    xg, s = _gpu_run(av, method, prob, 120, debugstep=10, dft=dft)
    assert rel(xg, xo) < REL_IMG, rel(xg, xo)
    st = s.stats()
    assert st.iterations == 120
    assert abs(st.sigma - tro["steps"][-1][0]) < 1e-5 * tro["steps"][-1][0]
    ex = s.export()
    gaps = ex["PDGap"].real
    assert len(gaps) == len(tro["PDGap"])
    assert np.allclose(gaps, tro["PDGap"], rtol=2e-4)
    if method == "ICTGV2":
        assert "x3_component" in ex
        assert np.allclose(ex["ICTGVnorm"].real, tro["ICTGVnorm"], rtol=2e-4)
        assert np.allclose(ex["DATAfidelity"].real, tro["DATAfidelity"], rtol=2e-4)
    if method == "ICTV":
        T, _, H, W = prob["kdata"].shape
        assert rel(ex["x3_component"].reshape(T, H, W), tro["x3"]) < REL_IMG
        assert np.allclose(ex["ictvnorm"].real, tro["ictvnorm"], rtol=2e-4)
        assert np.allclose(ex["DATAfidelity"].real, tro["DATAfidelity"], rtol=2e-4)
    if method in ("TV", "TVTEMP", "TGV2"):
        assert "x3_component" not in ex


@pytest.mark.parametrize("method,stop", [("TV", 2e-3), ("TVTEMP", 0.3), ("TGV2", 6e-3), ("ICTV", 0.5),
                                         ("ICTGV2", 7e-2)])
def test_stop_criterion(av, method, stop):
    """stopPDGap ends the loop at the same gap evaluation as the oracle
    (tv.cpp:186-190, tv_temp.cpp:174-175, tgv2.cpp:325-326, ictv.cpp:362-363,
    ictgv2.cpp:481-482).  The TVtemp and ICTV gaps rise from their first
    evaluation on these problems (TVtemp's gap carries the spatial TV norm
    its regulariser does not penalise; ICTV's step rule leaves out the
    regulariser operators), so their thresholds end the loop at k = 0."""
    from avionic_b200 import synth
    prob = synth.small(5)
    xo, tro, _ = _oracle_run(method, prob, 400, stop=stop)
    assert tro["iterations"] < 400  # the threshold is reached
    xg, s = _gpu_run(av, method, prob, 400, stop=stop)
    st = s.stats()
    assert st.stopped_by_gap == 1
    assert st.iterations == tro["iterations"] + 1
    assert rel(xg, xo) < REL_IMG


@pytest.mark.parametrize("method", ["TV", "TGV2", "ICTGV2"])
def test_relative_stop(av, method):
    """avx_solver_set_relative_stop ends the loop at the first gap evaluation
    (every 20 iterations) whose gap is at most rel times the first gap; rel is
    placed between two evaluations of the oracle's gap history."""
    from avionic_b200 import synth
    prob = synth.small(6)
    _, tro, _ = _oracle_run(method, prob, 400, debugstep=20)
    r = np.asarray(tro["PDGap"]) / tro["PDGap"][0]
    run_min = np.minimum.accumulate(r)
    js = [j for j in range(3, len(r)) if r[j] < 0.98 * run_min[j - 1]]
    assert js, "the oracle's gap does not fall"
    j = js[0]
    rel_stop = float(np.sqrt(run_min[j - 1] * r[j]))
    import torch
    T, C, H, W = prob["kdata"].shape
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    s = av.Solver(method, op)
    p = s.params
    p.maxIt = 400
    s.params = p
    s.set_relative_stop(rel_stop)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))
    st = s.stats()
    assert st.stopped_by_gap == 1
    assert st.iterations == 20 * j + 1
    xo, _, _ = _oracle_run(method, prob, 20 * j + 1)
    assert rel(x.cpu().numpy(), xo) < REL_IMG


def test_tv_ellipses_128_full(av):
    """The TV benchmark problem (128x128, 20 frames, 8 coils, 500 iterations)."""
    from avionic_b200 import synth
    prob = synth.tv_ellipses_128(0)
    u0 = synth.time_average_u0(prob["kdata"], prob["mask"], prob["b1"])
    xo, _, _ = _oracle_run("TV", prob, 500, u0=u0)
    xg, _ = _gpu_run(av, "TV", prob, 500, u0=u0)
    assert rel(xg, xo) < REL_IMG, rel(xg, xo)


def test_reconstruct_host_matches_device_path(av):
    from avionic_b200 import synth
    prob = synth.small(3)
    p = av.default_params(av.TGV2)
    p.maxIt = 60
    x, st = av.reconstruct_host("TGV2", prob["kdata"], prob["mask"], prob["b1"], params=p)
    xo, _, _ = _oracle_run("TGV2", prob, 60)
    assert rel(x, xo) < REL_IMG
    assert st.iterations == 60


def test_reconstruct_host_reuses_state_correctly(av):
    """Repeated host calls (the kept operator/solver/graphs) give the same image
    as the first call, and a changed mask or parameter set rebuilds the state."""
    from avionic_b200 import synth
    prob = synth.small(4)
    p = av.default_params(av.TGV2)
    p.maxIt = 40
    x1, _ = av.reconstruct_host("TGV2", prob["kdata"], prob["mask"], prob["b1"], params=p)
    x2, _ = av.reconstruct_host("TGV2", prob["kdata"], prob["mask"], prob["b1"], params=p)
    assert np.array_equal(x1, x2)
    # another mask: must match the oracle for that mask, not the cached one
    prob2 = dict(prob)
    m2 = prob["mask"].copy()
    m2[:, 1::3, :] = 0.0
    prob2["mask"] = m2
    prob2["kdata"] = prob["kdata"] * m2[:, None]
    x3, _ = av.reconstruct_host("TGV2", prob2["kdata"], prob2["mask"], prob2["b1"], params=p)
    xo, _, _ = _oracle_run("TGV2", prob2, 40)
    assert rel(x3, xo) < REL_IMG
    # another lambda
    q = av.default_params(av.TGV2)
    q.maxIt = 40
    q.adaptLambda = 0
    q.lambda_ = 3.0
    x4, _ = av.reconstruct_host("TGV2", prob["kdata"], prob["mask"], prob["b1"], params=q)
    assert rel(x4, x1) > 1e-4
    av.lib.avx_reconstruct_host_release()


def test_split_dft_matches_fp32_cine_192_shape(av):
    """The split-BF16x3 tensor-core y-transform agrees with the fp32 CUDA-core
    one at the benchmark shape (192 x 192, 16 coils, 16 rows per frame)."""
    import torch
    from avionic_b200 import synth
    prob = synth.cine_192(2, T=4)
    T, C, H, W = prob["kdata"].shape
    rng = np.random.default_rng(3)
    x = av.to_device(cplx(rng, (T, H, W)))
    b1 = av.to_device(prob["b1"])
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    assert op.dft_mode == av.DFT_SPLIT_BF16X3
    ks = op.backward(x, b1).cpu().numpy()
    op.dft_mode = av.DFT_FP32
    kf = op.backward(x, b1).cpu().numpy()
    oop = OCart(W, H, C, T, mask=prob["mask"], centered=False)
    ko = oop.backward(x.cpu().numpy().astype(complex), prob["b1"].astype(complex))
    assert rel(kf, ko) < REL_OP
    assert rel(ks, ko) < REL_OP
    # the adjoint (column transform + coil combine) in both forms
    z = cplx(rng, (T, C, H, W)) * prob["mask"][:, None]
    io = oop.forward(z.astype(complex), prob["b1"].astype(complex))
    op.dft_mode = av.DFT_SPLIT_BF16X3
    i_s = op.forward(av.to_device(z), b1).cpu().numpy()
    op.dft_mode = av.DFT_FP32
    i_f = op.forward(av.to_device(z), b1).cpu().numpy()
    assert rel(i_f, io) < REL_OP
    assert rel(i_s, io) < REL_OP
    torch.cuda.synchronize()
