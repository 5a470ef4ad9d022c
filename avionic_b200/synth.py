"""Seeded synthetic Cartesian 2D+t problems (stand-ins for the reference's
public cine / perfusion data, which are not available here).

Shapes and value distributions follow the benchmark configurations:

* ``config0``: 128x128, 20 frames, 8 coils; three ellipses whose radii
  oscillate with period 20 frames, smooth random phase; Gaussian-decay coil
  maps from 8 centres on a circle of radius 0.8 FOV (sigma 0.4 FOV) times a
  linear phase; per-frame mask of the 8 central phase-encode lines plus random
  lines to acceleration 8; complex Gaussian noise at 1e-3 of max |k|.
* ``config1``: 192x192, 30 frames, 16 coils; beating ring and blood-pool disc
  (radius factor 1 + 0.15 sin(2 pi t / 30)) over a static textured background
  of smoothed uniform noise; variable-density phase-encode lines (Gaussian
  line density, sigma 0.25 N) at acceleration 12, shifted per frame.
* ``batched``: sizes drawn from the seed as in the batched configuration.

k-space is formed with the library's operator convention: the unitary 2D
transform with the e^{+2 pi i} kernel from image to k-space (numpy ``ifft2``
with ``norm="ortho"``), masked per frame; the phase-encode direction is y
(height), lines are constant along x (readout).
"""

import numpy as np


def _smooth(rng, shape, sigma_px):
    """Low-pass Gaussian-filtered white noise (FFT filter), unit max."""
    H, W = shape
    n = rng.standard_normal((H, W))
    ky = np.fft.fftfreq(H)[:, None]
    kx = np.fft.fftfreq(W)[None, :]
    filt = np.exp(-2.0 * (np.pi * sigma_px) ** 2 * (kx ** 2 + ky ** 2))
    s = np.real(np.fft.ifft2(np.fft.fft2(n) * filt))
    return s / (np.max(np.abs(s)) + 1e-30)


def coil_maps(H, W, C, rng):
    """Gaussian-decay magnitudes from C centres on a circle of radius
    0.8 FOV (sigma 0.4 FOV), times a linear phase; normalised so that
    sum_c |b_c|^2 = 1 at every pixel."""
    yy, xx = np.meshgrid(np.linspace(-1, 1, H), np.linspace(-1, 1, W), indexing="ij")
    b = np.empty((C, H, W), dtype=np.complex128)
    for c in range(C):
        ang = 2 * np.pi * c / C
        cy, cx = 0.8 * np.sin(ang), 0.8 * np.cos(ang)
        mag = np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * 0.4 ** 2))
        kx, ky = rng.uniform(-1.5, 1.5, size=2)
        b[c] = mag * np.exp(1j * np.pi * (kx * xx + ky * yy))
    b /= np.sqrt(np.sum(np.abs(b) ** 2, axis=0, keepdims=True))
    return b


def phantom_ellipses(H, W, T, rng, period=20):
    yy, xx = np.meshgrid(np.linspace(-1, 1, H), np.linspace(-1, 1, W), indexing="ij")
    phase = np.pi * _smooth(rng, (H, W), sigma_px=max(H, W) / 8)
    ell = [(0.0, 0.0, 0.7, 0.85, 1.0, 0.10), (0.2, -0.15, 0.25, 0.3, 0.6, 0.25), (-0.3, 0.25, 0.15, 0.2, 0.8, 0.3)]
    x = np.zeros((T, H, W), dtype=np.complex128)
    for t in range(T):
        img = np.zeros((H, W))
        for (cy, cx, ry, rx, val, amp) in ell:
            f = 1.0 + amp * np.sin(2 * np.pi * t / period)
            img += val * ((((yy - cy) / (ry * f)) ** 2 + ((xx - cx) / (rx * f)) ** 2) <= 1.0)
        x[t] = img * np.exp(1j * phase)
    return x


def phantom_cine(H, W, T, rng, period=30):
    yy, xx = np.meshgrid(np.linspace(-1, 1, H), np.linspace(-1, 1, W), indexing="ij")
    bg = 0.3 * (0.5 + 0.5 * _smooth(rng, (H, W), sigma_px=max(H, W) / 32))
    bg *= (yy ** 2 + xx ** 2) <= 0.95 ** 2
    x = np.zeros((T, H, W), dtype=np.complex128)
    r = np.sqrt(yy ** 2 + xx ** 2)
    for t in range(T):
        f = 1.0 + 0.15 * np.sin(2 * np.pi * t / period)
        pool = 1.0 * (r <= 0.25 * f)
        ring = 0.6 * ((r > 0.25 * f) & (r <= 0.25 * f + 0.12))
        x[t] = np.where(pool + ring > 0, pool + ring, bg)
    return x.astype(np.complex128)


def mask_central_random(H, W, T, R, ncenter, rng):
    """Per frame: the ncenter central phase-encode lines plus uniformly random
    lines up to H/R lines, reseeded per frame; lines constant along x."""
    m = np.zeros((T, H, W), dtype=np.float32)
    nl = max(ncenter, int(round(H / R)))
    c0 = H // 2 - ncenter // 2
    for t in range(T):
        rows = set(range(c0, c0 + ncenter))
        rest = [y for y in range(H) if y not in rows]
        rows |= set(rng.choice(rest, size=nl - len(rows), replace=False).tolist())
        m[t, sorted(rows), :] = 1.0
    return m


def mask_variable_density(H, W, T, R, rng, sigma_frac=0.25):
    """Variable-density phase-encode lines: H/R lines per frame drawn without
    replacement from a Gaussian line density (sigma = sigma_frac * H) centred
    on k-space centre, with the pattern shifted per frame."""
    m = np.zeros((T, H, W), dtype=np.float32)
    nl = max(1, int(round(H / R)))
    ky = np.fft.fftshift(np.arange(H) - H // 2)  # frequency of each stored row
    dens = np.exp(-0.5 * (ky / (sigma_frac * H)) ** 2)
    base = rng.choice(H, size=nl, replace=False, p=dens / dens.sum())
    for t in range(T):
        rows = (np.sort(base) + t) % H
        m[t, rows, :] = 1.0
    return m


def simulate(x, b1, mask, rng, noise_rel):
    """k[t,c] = mask[t] * (F(b1[c] x[t]) + noise), F unitary with e^{+2 pi i}."""
    k = np.fft.ifft2(b1[None, :, :, :] * x[:, None, :, :], norm="ortho")
    sd = noise_rel * np.max(np.abs(k))
    k = k + sd / np.sqrt(2) * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape))
    return k * mask[:, None, :, :]


def config0(seed=0, H=128, W=128, T=20, C=8):
    rng = np.random.default_rng(seed)
    x = phantom_ellipses(H, W, T, rng, period=20)
    b1 = coil_maps(H, W, C, rng)
    mask = mask_central_random(H, W, T, R=8, ncenter=8, rng=rng)
    k = simulate(x, b1, mask, rng, 1e-3)
    return dict(kdata=k.astype(np.complex64), mask=mask, b1=b1.astype(np.complex64), truth=x.astype(np.complex64))


def config1(seed=1, H=192, W=192, T=30, C=16):
    rng = np.random.default_rng(seed)
    x = phantom_cine(H, W, T, rng, period=30)
    b1 = coil_maps(H, W, C, rng)
    mask = mask_variable_density(H, W, T, R=12, rng=rng)
    k = simulate(x, b1, mask, rng, 1e-3)
    return dict(kdata=k.astype(np.complex64), mask=mask, b1=b1.astype(np.complex64), truth=x.astype(np.complex64))


def small(seed, H=24, W=20, T=6, C=4, R=4, binary=True):
    """A small random problem of the same kind, for parity tests."""
    rng = np.random.default_rng(seed)
    x = phantom_ellipses(H, W, T, rng, period=T)
    b1 = coil_maps(H, W, C, rng)
    mask = mask_central_random(H, W, T, R=R, ncenter=2, rng=rng)
    if not binary:
        mask = mask * rng.uniform(0.5, 1.5, size=mask.shape).astype(np.float32)
    k = simulate(x, b1, mask, rng, 1e-3)
    return dict(kdata=k.astype(np.complex64), mask=mask, b1=b1.astype(np.complex64), truth=x.astype(np.complex64))


def time_average_u0(kdata, mask, b1):
    """Initial image: coil-combined zero-filled time average (one frame)."""
    ksum = kdata.sum(axis=0)
    cnt = np.maximum(mask.sum(axis=0), 1.0)
    img = np.fft.fft2(ksum / cnt[None], norm="ortho")
    return np.sum(np.conj(b1) * img, axis=0).astype(np.complex64)
