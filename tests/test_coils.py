"""Coil-sensitivity estimation on the device: the reference's known answers
(CUDA/test/coil_construction.cc) through the C ABI, and parity with the
float64 oracle (oracle/coils.py) on a seeded synthetic problem."""

import numpy as np
import pytest

from tests import kat_inputs as ki

pytestmark = pytest.mark.gpu
EPS = 1e-3


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def test_coil_construction_kats_on_device(av, kats):
    import torch
    k = kats["coil_construction"]
    W, H, T = k["dims"]
    C = k["coils"]
    kd = av.to_device(ki.kspace(W, H, C, T))
    mask = av.to_device(np.ones((T, H, W)))
    u, crec = av.coil_time_averaged(kd, mask)
    uh, ch = u.cpu().numpy(), crec.cpu().numpy()
    for (x, y), want in k["time_averaged_u_real"]:
        assert abs(uh[y, x].real - want) < EPS
    for (x, y, c), want in k["time_averaged_crec_real"]:
        assert abs(ch[c, y, x].real - want) < EPS
    ua = torch.abs(u).to(torch.complex64).contiguous()
    b1 = av.coil_b1_from_u_h1(ua, crec)
    bh = b1.cpu().numpy()
    for (x, y, c), want in k["h1_abs_b1"]:
        assert abs(abs(bh[c, y, x]) - want) < EPS
    mi = int(np.argmax([np.sum(np.abs(ch[c])) for c in range(C)]))
    assert mi == k["initial_index"]
    uM = torch.zeros((H, W), dtype=torch.complex64, device="cuda")
    av.coil_utgv2(b1[mi:mi + 1].contiguous(), crec[mi:mi + 1].contiguous(), [0], uM)
    um = uM.cpu().numpy()
    for (x, y), want in k["utgv2_u_real"]:
        assert abs(um[y, x].real - want) < EPS
    x1 = av.coil_b1_recon((b1[1] * uM).contiguous(), crec[1:2].contiguous(), 1)
    bb = bh[1] * np.exp(1j * np.angle(x1.cpu().numpy()[0]))
    for (x, y), want in k["b1recon_coil1_real"]:
        assert abs(bb[y, x].real - want) < EPS
    uu, b1f = av.coil_construction(kd, mask)
    uu, b1f = uu.cpu().numpy(), b1f.cpu().numpy()
    for (x, y, c), want in k["loop_b1_real"]:
        assert abs(b1f[c, y, x].real - want) < EPS
    for (x, y, c), want in k["loop_u_real"]:
        assert abs(uu[c, y, x].real - want) < EPS


def test_coil_construction_matches_oracle(av):
    from avionic_b200 import synth
    from oracle import coils as co
    prob = synth.small(9, H=24, W=20, T=6, C=4, R=3)
    p = co.default_params()
    p["uNrIt"], p["b1NrIt"], p["b1FinalNrIt"] = 40, 60, 80
    uo, bo = co.perform_coil_construction(prob["kdata"].astype(complex), prob["mask"].astype(float), p)
    q = av.coil_default_params()
    q.uNrIt, q.b1NrIt, q.b1FinalNrIt = 40, 60, 80
    ug, bg = av.coil_construction(av.to_device(prob["kdata"]), av.to_device(prob["mask"]), q)
    ug, bg = ug.cpu().numpy(), bg.cpu().numpy()
    assert np.linalg.norm(bg - bo) / np.linalg.norm(bo) < 1e-4
    assert np.linalg.norm(ug - uo) / np.linalg.norm(uo) < 1e-4


def test_radial_coil_construction_matches_oracle(av):
    from oracle import coils as co
    from tests.test_radial import _problem
    pr = _problem(12, W=20, H=20, C=3, T=3, nfe=40, spf=7)
    p = co.default_params()
    p["uNrIt"], p["b1NrIt"], p["b1FinalNrIt"] = 30, 40, 50
    k = pr["k"].astype(np.complex64)
    traj = pr["traj"].astype(np.float32)
    dens = pr["dens"].astype(np.float32)
    uo, co_ = co.time_averaged_radial(k.astype(complex), traj.astype(float), dens.astype(float), pr["W"], pr["H"])
    S = traj.shape[2]
    import ctypes
    import torch
    u = torch.empty((pr["H"], pr["W"]), dtype=torch.complex64, device="cuda")
    crec = torch.empty((pr["C"], pr["H"], pr["W"]), dtype=torch.complex64, device="cuda")
    dt, dd, dk = av.to_device(traj), av.to_device(dens), av.to_device(k)
    av.check(av.lib.avx_coil_time_averaged_radial(pr["W"], pr["H"], pr["C"], pr["T"], S, av._cptr(dt), av._cptr(dd),
                                                  av._cptr(dk), av._cptr(u), av._cptr(crec), 1))
    assert np.linalg.norm(crec.cpu().numpy() - co_) / np.linalg.norm(co_) < 1e-5
    uo2, bo = co.estimate_from(uo, co_, p)
    q = av.coil_default_params()
    q.uNrIt, q.b1NrIt, q.b1FinalNrIt = 30, 40, 50
    ug = torch.empty((pr["C"], pr["H"], pr["W"]), dtype=torch.complex64, device="cuda")
    bg = torch.empty_like(ug)
    av.check(av.lib.avx_coil_construction_radial(pr["W"], pr["H"], pr["C"], pr["T"], S, ctypes.byref(q), av._cptr(dt),
                                                 av._cptr(dd), av._cptr(dk), av._cptr(ug), av._cptr(bg)))
    bg = bg.cpu().numpy()
    assert np.linalg.norm(bg - bo) / np.linalg.norm(bo) < 1e-4
