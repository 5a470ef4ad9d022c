"""The CLI's -o data normalisation (avx_normalize_data).

CPU tests pin the factor selection of FindNormalizationFactor
(raw_data_preparation.cpp:661-686) and utils::Median (utils.cpp:1442-1462) on
hand-made vectors; GPU tests compare the device normalisation (Cartesian with
even and odd sizes, radial) and the executable's -o run with the float64
oracle.
"""

import numpy as np
import pytest

from oracle.normalize import find_normalization_factor, normalization_factor


def test_factor_selection_follows_scan_order():
    # values >= 0.9 max before the first maximum are not collected
    assert find_normalization_factor([9.5, 9.6, 10.0, 1.0, 9.0, 2.0]) == pytest.approx(9.5)
    # odd count: the middle value
    assert find_normalization_factor([1.0, 10.0, 9.9, 9.1, 3.0]) == pytest.approx(9.9)
    # the first of several maxima starts the scan; 0.9 max itself is included
    assert find_normalization_factor([10.0, 9.0, 10.0, 8.99]) == pytest.approx(10.0)
    assert find_normalization_factor([0.0, 4.0]) == pytest.approx(4.0)


def _margin_ok(mag):
    """True when no value lies within 1e-5 (relative) of the 0.9 threshold,
    so FP32 and FP64 magnitudes select the same set."""
    v = np.asarray(mag).ravel()
    thr = 0.9 * v.max()
    return not np.any(np.abs(v - thr) <= 1e-5 * thr)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(24, 20), (15, 21)])
def test_cartesian_normalisation_matches_oracle(shape):
    import torch
    import avionic_b200 as av
    from avionic_b200 import synth
    from oracle.coils import time_averaged_reconstruction
    H, W = shape
    prob = synth.small(31, H=H, W=W)
    k64 = prob["kdata"].astype(complex)
    u, _ = time_averaged_reconstruction(k64, prob["mask"], centered=True, apply_phase=False)
    assert _margin_ok(np.abs(u))
    fo = normalization_factor(k64, prob["mask"])
    kd = torch.from_numpy(prob["kdata"]).cuda()
    md = torch.from_numpy(prob["mask"]).cuda()
    for _ in range(2):  # the same factor on a second call with fresh data
        k = kd.clone()
        f = av.normalize_data(k, md)
        assert abs(f - fo) / fo < 1e-5
        assert torch.allclose(k, kd * f, rtol=1e-6, atol=0)


@pytest.mark.gpu
def test_radial_normalisation_matches_oracle():
    import torch
    import avionic_b200 as av
    from oracle.coils import time_averaged_radial
    from tests.test_radial import _problem
    pr = _problem(17)
    k32 = pr["k"].astype(np.complex64)
    tr, de = pr["traj"].astype(np.float32), pr["dens"].astype(np.float32)
    u, _ = time_averaged_radial(k32.astype(complex), tr.astype(float), de.astype(float), pr["W"], pr["H"],
                                apply_phase=False)
    assert _margin_ok(np.abs(u))
    fo = normalization_factor(k32.astype(complex), traj=tr.astype(float), dens=de.astype(float), W=pr["W"],
                              H=pr["H"])
    kd = torch.from_numpy(k32).cuda()
    k = kd.clone()
    f = av.normalize_data(k, traj=torch.from_numpy(tr).cuda(), dens=torch.from_numpy(de).cuda(), width=pr["W"],
                          height=pr["H"])
    assert abs(f - fo) / fo < 1e-5
    assert torch.allclose(k, kd * f, rtol=1e-6, atol=0)


@pytest.mark.gpu
def test_zero_data_is_an_error():
    import torch
    import avionic_b200 as av
    k = torch.zeros((2, 2, 8, 8), dtype=torch.complex64, device="cuda")
    m = torch.ones((2, 8, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(av.AvionicError, match="normalisation"):
        av.normalize_data(k, m)
