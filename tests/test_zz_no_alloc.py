"""The TV norm entry point that allocates nothing (avx_tv_norm_noalloc).

It serves callers that cannot allocate device memory when they need the
result (fixed memory budgets, host bindings without a CUDA allocator); its
partial sums live in a fixed __device__ array.  This file is collected last
so that a failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AVX_E_ARG = 1
MAX_PIXELS = 2_097_152


@pytest.fixture(scope="module")
def av():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import avionic_b200
    return avionic_b200


def noalloc(av, u, w):
    T, H, W = u.shape
    out = ctypes.c_double(float("nan"))
    st = av.lib.avx_tv_norm_noalloc(ctypes.c_void_p(u.data_ptr()), W, H, T, w[0], w[1], w[2], ctypes.byref(out))
    return st, out.value


def test_noalloc_matches_allocating_entry_point_twice(av):
    rng = np.random.default_rng(2024)
    imgs = [
        (rng.standard_normal((20, 128, 128)) + 1j * rng.standard_normal((20, 128, 128))).astype(np.complex64),
        (rng.standard_normal((5, 13, 7)) + 1j * rng.standard_normal((5, 13, 7))).astype(np.complex64),
    ]
    weights = [(1.0, 1.0, 1.0), (1.2, 1.2, 2.0)]
    for u_np, w in zip(imgs, weights):  # two calls in a row on different inputs
        u = av.to_device(u_np)
        st, got = noalloc(av, u, w)
        assert st == 0, av.lib.avx_last_error()
        ref = av.tv_norm(u, *w)
        assert abs(got - ref) <= 1e-9 * abs(ref), (got, ref)


def test_noalloc_reference_kat(av, kats):
    """utils::TVNorm known answer (CUDA/test/tv.cc:293-319) through the no-alloc path."""
    from tests import kat_inputs as ki
    k = kats["tv_norm"]
    W, H, T = k["dims"]
    for case in k["cases"]:
        s = complex(case["scale"]) if isinstance(case["scale"], str) else case["scale"]
        st, got = noalloc(av, av.to_device(s * ki.image(W, H, T)), case["w"])
        assert st == 0
        assert abs(got - case["value"]) < max(1e-3, 2e-6 * case["value"])


def test_noalloc_rejects_sizes_beyond_its_scratch(av):
    import torch
    u = torch.zeros((1, 1, 1), dtype=torch.complex64, device="cuda")
    T, H, W = 1, 1024, MAX_PIXELS // 1024 + 1  # dimensions only; rejected before any launch
    out = ctypes.c_double(0.0)
    st = av.lib.avx_tv_norm_noalloc(ctypes.c_void_p(u.data_ptr()), W, H, T, 1.0, 1.0, 1.0, ctypes.byref(out))
    assert st == AVX_E_ARG
    assert b"scratch limit" in av.lib.avx_last_error()
