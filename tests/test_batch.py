"""Batch / serve engine (avx_batch_*): concurrent requests of mixed sizes,
methods and operators give the same images as single solver runs, the HBM
budget is enforced at submission, and completions carry their tags."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def _solo(av, method, prob, params):
    import torch
    T, C, H, W = prob["kdata"].shape
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    s = av.Solver(method, op, params)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))
    return x.cpu().numpy()


def test_batch_matches_single_runs(av):
    import torch
    from avionic_b200 import synth
    cases = [("TV", synth.small(21, H=24, W=20, T=6, C=4)), ("TGV2", synth.small(22, H=32, W=28, T=5, C=3)),
             ("ICTGV2", synth.small(23, H=20, W=24, T=4, C=5)), ("TGV2", synth.small(24, H=16, W=16, T=8, C=2)),
             ("TV", synth.small(25, H=40, W=36, T=3, C=6))]
    eng = av.BatchEngine(0, hbm_budget=4 << 30, workers=3)
    keep = []
    for i, (m, prob) in enumerate(cases):
        p = av.default_params(av.METHODS[m])
        p.maxIt = 60
        T, C, H, W = prob["kdata"].shape
        d, b1, mask = av.to_device(prob["kdata"]), av.to_device(prob["b1"]), av.to_device(prob["mask"])
        x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
        r = av.cartesian_request(m, d, x, b1, mask=mask, params=p, tag=100 + i)
        assert av.query_workspace(r) > 0
        eng.submit(r)
        keep.append((m, prob, p, x, d, b1, mask))
    got = {}
    while len(got) < len(cases):
        for c in eng.poll(wait_ms=-1):
            got[c.tag] = c
    assert eng.pending == 0
    for i, (m, prob, p, x, *_rest) in enumerate(keep):
        c = got[100 + i]
        assert c.status == 0
        assert c.stats.iterations == 60
        assert c.workspace_bytes > 0 and c.run_ms > 0
        want = _solo(av, m, prob, p)
        np.testing.assert_array_equal(x.cpu().numpy(), want)
    eng.close()


def test_batch_radial_request(av):
    import torch
    from tests.test_radial import _problem
    pr = _problem(31, W=20, H=20, C=3, T=3, nfe=40, spf=7)
    p = av.default_params(av.TGV2)
    p.maxIt = 40
    traj = av.to_device(pr["traj"].astype(np.float32))
    dens = av.to_device(pr["dens"].astype(np.float32))
    k = av.to_device(pr["k"].astype(np.complex64))
    b1 = av.to_device(pr["b1"].astype(np.complex64))
    x = torch.zeros((pr["T"], pr["H"], pr["W"]), dtype=torch.complex64, device="cuda")
    eng = av.BatchEngine(0, hbm_budget=1 << 30, workers=2)
    eng.submit(av.radial_request("TGV2", k, x, b1, traj, dens, pr["spf"], pr["nfe"], params=p, osf=2.0, tag=7))
    eng.drain()
    (c,) = eng.poll()
    assert c.tag == 7 and c.status == 0 and c.stats.iterations == 40
    op = av.RadialOperator(pr["W"], pr["H"], pr["C"], pr["T"], traj, dens, pr["spf"], 3.0, 8.0, 2.0)
    s = av.Solver("TGV2", op, p)
    x2 = torch.zeros_like(x)
    s.run(k, x2, b1)
    np.testing.assert_array_equal(x.cpu().numpy(), x2.cpu().numpy())
    eng.close()


def test_batch_budget_is_enforced(av):
    import torch
    from avionic_b200 import synth
    prob = synth.small(26)
    T, C, H, W = prob["kdata"].shape
    d, b1, mask = av.to_device(prob["kdata"]), av.to_device(prob["b1"]), av.to_device(prob["mask"])
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    r = av.cartesian_request("TV", d, x, b1, mask=mask)
    need = av.query_workspace(r)
    eng = av.BatchEngine(0, hbm_budget=need - 1, workers=1)
    with pytest.raises(av.AvionicError):
        eng.submit(r)
    assert eng.pending == 0
    eng.close()
    # a budget for one request at a time still completes several, one after another
    eng = av.BatchEngine(0, hbm_budget=need + 1, workers=4)
    xs = []
    for i in range(3):
        xi = torch.zeros_like(x)
        xs.append(xi)
        p = av.default_params(av.TV)
        p.maxIt = 20
        eng.submit(av.cartesian_request("TV", d, xi, b1, mask=mask, params=p, tag=i))
    eng.drain()
    cs = eng.poll(max_items=8)
    assert sorted(c.tag for c in cs) == [0, 1, 2]
    assert all(c.status == 0 for c in cs)
    np.testing.assert_array_equal(xs[0].cpu().numpy(), xs[2].cpu().numpy())
    eng.close()


def _radial_items(av, seed, W=20, H=20, C=3, T=3, nfe=40, spf=7):
    from tests.test_radial import _problem
    pr = _problem(seed, W=W, H=H, C=C, T=T, nfe=nfe, spf=spf)
    return dict(traj=av.to_device(pr["traj"].astype(np.float32)), dens=av.to_device(pr["dens"].astype(np.float32)),
                k=av.to_device(pr["k"].astype(np.complex64)), b1=av.to_device(pr["b1"].astype(np.complex64)),
                shape=(pr["T"], pr["H"], pr["W"]), spf=pr["spf"], nfe=pr["nfe"], C=pr["C"])


def _solo_radial(av, method, it, params):
    import torch
    T, H, W = it["shape"]
    op = av.RadialOperator(W, H, it["C"], T, it["traj"], it["dens"], it["spf"], 3.0, 8.0, 2.0)
    s = av.Solver(method, op, params)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    s.run(it["k"], x, it["b1"])
    return x.cpu().numpy(), s.stats()


def _solo_cart(av, method, prob, params, dft):
    import torch
    T, C, H, W = prob["kdata"].shape
    op = av.CartesianOperator(W, H, C, T, mask=av.to_device(prob["mask"]), centered=False)
    op.dft_mode = dft
    s = av.Solver(method, op, params)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    s.run(av.to_device(prob["kdata"]), x, av.to_device(prob["b1"]))
    return x.cpu().numpy(), s.stats()


def test_mixed_stream_is_the_same_alone_and_in_the_mix(av):
    """Cartesian requests in both forms of the y-transforms and radial
    requests, of every method, some submitted while the others already run:
    each image equals its request run alone, bit for bit."""
    import time

    import torch
    from avionic_b200 import synth
    eng = av.BatchEngine(0, hbm_budget=8 << 30, workers=6)
    reqs = []
    methods = ["TV", "TGV2", "ICTGV2", "TVTEMP", "ICTV"]
    for i in range(10):
        m = methods[i % len(methods)]
        p = av.default_params(av.METHODS[m])
        p.maxIt = 40 + 20 * (i % 3)
        if i % 3 == 2:
            it = _radial_items(av, 40 + i)
            T, H, W = it["shape"]
            x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
            r = av.radial_request(m, it["k"], x, it["b1"], it["traj"], it["dens"], it["spf"], it["nfe"], params=p,
                                  osf=2.0, tag=i)
            reqs.append(("radial", m, it, p, x, None))
        else:
            prob = synth.small(60 + i, H=24 + 4 * (i % 2), W=20, T=4 + i % 3, C=3)
            dft = av.DFT_SPLIT_BF16X3 if i % 2 == 0 else av.DFT_FP32
            T, C, H, W = prob["kdata"].shape
            d, b1, mask = av.to_device(prob["kdata"]), av.to_device(prob["b1"]), av.to_device(prob["mask"])
            x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
            r = av.cartesian_request(m, d, x, b1, mask=mask, params=p, dft_mode=dft, tag=i)
            reqs.append(("cart", m, prob, p, x, (d, b1, mask, dft)))
        eng.submit(r)
        if i == 4:
            time.sleep(0.05)  # the rest arrive while the first ones run
    got = {}
    while len(got) < len(reqs):
        for c in eng.poll(wait_ms=-1):
            got[c.tag] = c
    eng.close()
    for i, (kind, m, item, p, x, extra) in enumerate(reqs):
        c = got[i]
        assert c.status == 0, (i, c.status)
        if kind == "radial":
            want, st = _solo_radial(av, m, item, p)
        else:
            want, st = _solo_cart(av, m, item, p, extra[3])
            assert c.dft_mode == extra[3]
        assert c.stats.iterations == st.iterations == p.maxIt
        np.testing.assert_array_equal(x.cpu().numpy(), want)


@pytest.mark.parametrize("how", ["stopPDGap", "relative"])
def test_engine_retires_requests_at_their_stop_test(av, how):
    """The engine retires a request at the gap evaluation that ends the
    reference's loop (tgv2.cpp:317-330) or the relative test; the image and
    the iteration count equal the request run alone."""
    import torch
    from avionic_b200 import synth
    prob = synth.small(5)
    T, C, H, W = prob["kdata"].shape
    p = av.default_params(av.TGV2)
    p.maxIt = 400
    rel = 0.0
    if how == "stopPDGap":
        p.stopPDGap = 6e-3
    else:
        rel = 0.2
    d, b1, mask = av.to_device(prob["kdata"]), av.to_device(prob["b1"]), av.to_device(prob["mask"])
    eng = av.BatchEngine(0, hbm_budget=2 << 30, workers=2)
    x = torch.zeros((T, H, W), dtype=torch.complex64, device="cuda")
    eng.submit(av.cartesian_request("TGV2", d, x, b1, mask=mask, params=p, tag=1, stop_gap_rel=rel))
    (c,) = eng.poll(wait_ms=-1)
    eng.close()
    assert c.status == 0 and c.stats.stopped_by_gap == 1 and c.stats.iterations < 400
    op = av.CartesianOperator(W, H, C, T, mask=mask, centered=False)
    s = av.Solver("TGV2", op, p)
    if rel > 0:
        s.set_relative_stop(rel)
    x2 = torch.zeros_like(x)
    s.run(d, x2, b1)
    assert s.stats().iterations == c.stats.iterations
    np.testing.assert_array_equal(x.cpu().numpy(), x2.cpu().numpy())
