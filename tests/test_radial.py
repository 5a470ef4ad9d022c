"""Radial (gridding) operator: oracle properties on CPU, device parity on GPU.

The reference's radial arithmetic lives in gpuNUFFT, which is not in the tree,
so its golden values (CUDA/test/noncartesian_operator.cc:120-158) cannot be
reproduced; parity is against the float64 oracle of the same gridding
definition (oracle/radial.py), plus adjointness and the approximation error
against the exact non-uniform DFT.
"""

import numpy as np
import pytest

from oracle import radial as rd
from oracle import solvers as so


def _problem(seed, W=24, H=20, C=3, T=3, nfe=48, spf=9, osf=1.5):
    rng = np.random.default_rng(seed)
    traj, dens = rd.golden_angle_radial(nfe, spf, T)
    yy, xx = np.meshgrid(np.linspace(-1, 1, H), np.linspace(-1, 1, W), indexing="ij")
    x = np.zeros((T, H, W), complex)
    for t in range(T):
        x[t] = ((yy / (0.6 + 0.05 * t)) ** 2 + (xx / 0.7) ** 2 <= 1) * np.exp(0.3j * xx)
    b1 = rng.standard_normal((C, H, W)) + 1j * rng.standard_normal((C, H, W))
    b1 /= np.sqrt(np.sum(np.abs(b1) ** 2, axis=0, keepdims=True))
    k = np.zeros((T, C, traj.shape[2]), complex)
    for t in range(T):
        for c in range(C):
            k[t, c] = rd.nudft(b1[c] * x[t], traj[t]) / np.sqrt(W * H)
    k = k + 1e-3 * np.max(np.abs(k)) * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape))
    k *= np.sqrt(dens)[:, None, :]  # the data are sqrt(w)-weighted, as main.cpp:546-570 does
    return dict(W=W, H=H, C=C, T=T, nfe=nfe, spf=spf, osf=osf, traj=traj, dens=dens, x=x, b1=b1, k=k)


def test_oracle_adjoint_and_accuracy():
    p = _problem(0)
    op = rd.RadialOperator(p["W"], p["H"], p["C"], p["T"], p["traj"], p["dens"], 3.0, 8.0, 2.0)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((p["T"], p["H"], p["W"])) + 1j * rng.standard_normal((p["T"], p["H"], p["W"]))
    z = rng.standard_normal((p["T"], p["C"], op.S)) + 1j * rng.standard_normal((p["T"], p["C"], op.S))
    lhs = np.vdot(op.backward(x, p["b1"]), z)
    rhs = np.vdot(x, op.forward(z, p["b1"]))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12
    # approximation error of the gridding against the exact NUDFT (J = 3, osf 2)
    u = p["b1"][0] * x[0]
    exact = rd.nudft(u, p["traj"][0])
    approx = op.backward(x, p["b1"])[0, 0] / op.sqrt_w[0] / op.norm
    assert np.linalg.norm(approx - exact) / np.linalg.norm(exact) < 0.02


def test_oracle_sector_map_is_a_partition():
    p = _problem(2)
    G = (rd.grid_size(p["H"], 1.5), rd.grid_size(p["W"], 1.5))
    order, start = rd.sector_map(p["traj"], G, 8.0)
    for f in range(p["T"]):
        assert np.array_equal(np.sort(order[f]), np.arange(p["traj"].shape[2]))
        assert start[f, -1] == p["traj"].shape[2] and np.all(np.diff(start[f]) >= 0)


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


def _ops(av, p, osf=None):
    osf = osf or p["osf"]
    g = av.RadialOperator(p["W"], p["H"], p["C"], p["T"], av.to_device(p["traj"].astype(np.float32)),
                          av.to_device(p["dens"].astype(np.float32)), p["spf"], 3.0, 8.0, osf)
    o = rd.RadialOperator(p["W"], p["H"], p["C"], p["T"], p["traj"].astype(np.float32).astype(float),
                          p["dens"].astype(np.float32).astype(float), 3.0, 8.0, osf)
    return g, o


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.gpu
@pytest.mark.parametrize("osf", [1.5, 2.0])
def test_radial_operator_matches_oracle(av, osf):
    import ctypes
    p = _problem(3)
    g, o = _ops(av, p, osf)
    rng = np.random.default_rng(4)
    x = (rng.standard_normal((p["T"], p["H"], p["W"])) + 1j * rng.standard_normal((p["T"], p["H"], p["W"])))
    z = rng.standard_normal((p["T"], p["C"], o.S)) + 1j * rng.standard_normal((p["T"], p["C"], o.S))
    b1 = p["b1"].astype(np.complex64)
    kg = g.backward(av.to_device(x.astype(np.complex64)), av.to_device(b1)).cpu().numpy()
    ko = o.backward(x.astype(np.complex64).astype(complex), b1.astype(complex))
    assert rel(kg, ko) < 1e-5
    ig = g.forward(av.to_device(z.astype(np.complex64)), av.to_device(b1)).cpu().numpy()
    io = o.forward(z.astype(np.complex64).astype(complex), b1.astype(complex))
    assert rel(ig, io) < 1e-5
    # adjointness of the device pair
    lhs = np.vdot(kg.astype(complex), z.astype(np.complex64).astype(complex))
    rhs = np.vdot(x.astype(np.complex64).astype(complex), ig.astype(complex))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    # sector layout: bit-exact against the oracle's float32 computation
    S = o.S
    nsx, nsy = int(np.ceil(o.Gx / 8)), int(np.ceil(o.Gy / 8))
    order = np.zeros(p["T"] * S, np.int32)
    start = np.zeros(p["T"] * (nsx * nsy + 1), np.int32)
    gxy = np.zeros(2, np.int32)
    av.check(av.lib.avx_radial_sector_map(g.handle, order.ctypes.data_as(ctypes.c_void_p),
                                          start.ctypes.data_as(ctypes.c_void_p), gxy.ctypes.data_as(ctypes.c_void_p)))
    assert (gxy[0], gxy[1]) == (o.Gx, o.Gy)
    oo, os_ = rd.sector_map(p["traj"].astype(np.float32), (o.Gy, o.Gx), 8.0)
    assert np.array_equal(order.reshape(p["T"], S), oo)
    assert np.array_equal(start.reshape(p["T"], -1), os_)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["TV", "TGV2", "ICTGV2"])
def test_radial_solver_matches_oracle(av, method):
    import torch
    p = _problem(5)
    g, o = _ops(av, p)
    q = so.init_params(method)
    q.maxIt, q.lam = 60, 4.0
    q.debug, q.debugstep = True, 10
    tr = {}
    xo = so.run(method, p["k"].astype(np.complex64).astype(complex), np.zeros((p["T"], p["H"], p["W"]), complex),
                p["b1"].astype(np.complex64).astype(complex), o, q, tr)
    params = av.default_params(av.METHODS[method])
    params.maxIt, params.lambda_, params.adaptLambda = 60, 4.0, 0
    s = av.Solver(method, g, params)
    s.set_debug(True, 10)
    x = torch.zeros((p["T"], p["H"], p["W"]), dtype=torch.complex64, device="cuda")
    s.run(av.to_device(p["k"].astype(np.complex64)), x, av.to_device(p["b1"].astype(np.complex64)))
    assert rel(x.cpu().numpy(), xo) < 1e-4
    gaps = s.export()["PDGap"].real
    assert np.allclose(gaps, tr["PDGap"], rtol=1e-3)


@pytest.mark.gpu
def test_radial_adapt_lambda(av):
    p = _problem(6)
    g, o = _ops(av, p)
    assert abs(g.adapt_lambda(0.34, 4.57) - o.adapt_lambda(0.34, 4.57, p["spf"])) < 1e-5


@pytest.mark.gpu
def test_trajectory_outside_the_grid_is_rejected():
    """Window offsets are wrapped once; a trajectory beyond +-1/2 cycle/pixel is refused."""
    import torch
    import avionic_b200 as av
    p = _problem(3)
    tr = torch.from_numpy(p["traj"].astype(np.float32)).cuda()
    de = torch.from_numpy(p["dens"].astype(np.float32)).cuda()
    tr[0, 0, 5] = 0.6
    with pytest.raises(av.AvionicError, match="trajectory"):
        av.RadialOperator(p["W"], p["H"], p["C"], p["T"], tr, de, p["spf"], 3.0, 8.0, 1.5)
