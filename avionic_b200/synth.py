"""Seeded synthetic Cartesian 2D+t problems (stand-ins for the reference's
public cine / perfusion data, which are not available here).

Shapes and value distributions follow the benchmark problems:

* ``tv_ellipses_128``: 128x128, 20 frames, 8 coils; three ellipses whose radii
  oscillate with period 20 frames, smooth random phase; Gaussian-decay coil
  maps from 8 centres on a circle of radius 0.8 FOV (sigma 0.4 FOV) times a
  linear phase; per-frame mask of the 8 central phase-encode lines plus random
  lines to acceleration 8; complex Gaussian noise at 1e-3 of max |k|.
* ``cine_192``: 192x192, 30 frames, 16 coils; beating ring and blood-pool disc
  (radius factor 1 + 0.15 sin(2 pi t / 30)) over a static textured background
  of smoothed uniform noise; variable-density phase-encode lines (Gaussian
  line density, sigma 0.25 N) at acceleration 12, shifted per frame.
* ``batched_specs`` / ``cine_instance_gpu``: 64 instances of uneven size
  (matrix uniform in {96, 128, 160, 192, 256, 320}, frames 8-48, coils 4-32,
  acceleration 6-16), each generated as ``cine_192`` from its own seed, with
  the k-space formed on the GPU (torch.fft) so that large instances are quick.
* ``radial_128_gpu``: radial golden-angle acquisition of the ``cine_192`` phantom
  at 128 x 128 (256 readout samples, 21 spokes per frame, 40 frames, 12
  coils); k-space by an exact float64 non-uniform DFT on the GPU, complex
  Gaussian noise at 2e-3 of max |k|, sqrt(w)-weighted as the CLI weights it.
* ``serving_stream``: a Poisson arrival stream mixing TV / TGV2 / ICTGV2 (50 /
  30 / 20 %) and Cartesian (batched sizes) / radial (128 x 128 image, 256
  readout samples, 13-34 golden-angle spokes per frame, 20-60 frames, 12
  coils) requests (70 / 30 %).

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


def tv_ellipses_128(seed=0, H=128, W=128, T=20, C=8):
    rng = np.random.default_rng(seed)
    x = phantom_ellipses(H, W, T, rng, period=20)
    b1 = coil_maps(H, W, C, rng)
    mask = mask_central_random(H, W, T, R=8, ncenter=8, rng=rng)
    k = simulate(x, b1, mask, rng, 1e-3)
    return dict(kdata=k.astype(np.complex64), mask=mask, b1=b1.astype(np.complex64), truth=x.astype(np.complex64))


def cine_192(seed=1, H=192, W=192, T=30, C=16):
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


# ---------------------------------------------------------------------------
# batched and served workloads
# ---------------------------------------------------------------------------

MATRICES = (96, 128, 160, 192, 256, 320)


def batched_specs(seed=3, n=64):
    """Sizes of the batched configuration, one dict per instance."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        m = int(rng.choice(MATRICES))
        out.append(dict(W=m, H=m, T=int(rng.integers(8, 49)), C=int(rng.integers(4, 33)),
                        R=int(rng.integers(6, 17)), seed=int(rng.integers(1 << 31))))
    return out


def cine_instance_gpu(spec, device="cuda", noise_rel=1e-3):
    """A ``cine_192``-style instance at spec's sizes: returns CUDA tensors
    kdata (T,C,H,W) masked, mask (T,H,W), b1 (C,H,W) and x0 (T,H,W), the
    coil-combined zero-filled time average replicated over the frames."""
    import torch
    H, W, T, C = spec["H"], spec["W"], spec["T"], spec["C"]
    rng = np.random.default_rng(spec["seed"])
    x = torch.from_numpy(phantom_cine(H, W, T, rng, period=30).astype(np.complex64)).to(device)
    b1 = torch.from_numpy(coil_maps(H, W, C, rng).astype(np.complex64)).to(device)
    mask = torch.from_numpy(mask_variable_density(H, W, T, R=spec["R"], rng=rng)).to(device)
    k = torch.empty((T, C, H, W), dtype=torch.complex64, device=device)
    for t in range(T):
        k[t] = torch.fft.ifft2(b1 * x[t], norm="ortho")
    sd = noise_rel * float(k.abs().max())
    g = torch.Generator(device=device)
    g.manual_seed(spec["seed"])
    k += (sd / np.sqrt(2.0)) * torch.complex(torch.randn(k.shape, generator=g, device=device),
                                            torch.randn(k.shape, generator=g, device=device))
    k *= mask[:, None]
    cnt = torch.clamp(mask.sum(0), min=1.0)
    img = torch.fft.fft2(k.sum(0) / cnt[None], norm="ortho")
    u0 = (b1.conj() * img).sum(0)
    x0 = u0[None].repeat(T, 1, 1).contiguous()
    return dict(kdata=k, mask=mask, b1=b1, x0=x0)


def golden_angle_radial(n_ro, spokes_per_frame, frames, angle_deg=111.246117975):
    """Golden-angle radial trajectory (T, 2, S) float32 in [-0.5, 0.5) and a
    ramp density (T, S) normalised to max 1; S = n_ro * spokes_per_frame."""
    r = (np.arange(n_ro) - n_ro / 2.0) / n_ro
    th = np.deg2rad(angle_deg) * np.arange(frames * spokes_per_frame).reshape(frames, spokes_per_frame)
    kx = (np.cos(th)[:, :, None] * r[None, None, :]).reshape(frames, -1)
    ky = (np.sin(th)[:, :, None] * r[None, None, :]).reshape(frames, -1)
    traj = np.stack([kx, ky], axis=1).astype(np.float32)
    dens = np.broadcast_to(np.abs(r) + 0.5 / n_ro, (frames, spokes_per_frame, n_ro)).reshape(frames, -1)
    dens = (dens / dens.max()).astype(np.float32)
    return traj, dens


def radial_instance_gpu(spec, device="cuda", noise_rel=2e-3, kernel_width=3.0, sector_width=8.0, osf=1.5):
    """A radial instance: the ``cine_192`` phantom at spec's image size, coil
    maps as ``coil_maps``, golden-angle spokes; k-space = the library's radial
    operator applied to the phantom (sqrt(w)-weighted, as the solver expects)
    plus complex Gaussian noise.  Returns CUDA tensors kdata (T,C,S), traj,
    dens, b1, x0 (zeros) and the sample counts."""
    import torch
    import avionic_b200 as av
    H, W, T, C = spec["H"], spec["W"], spec["T"], spec["C"]
    nfe, spf = spec["n_fe"], spec["spokes"]
    rng = np.random.default_rng(spec["seed"])
    x = torch.from_numpy(phantom_cine(H, W, T, rng, period=30).astype(np.complex64)).to(device)
    b1 = torch.from_numpy(coil_maps(H, W, C, rng).astype(np.complex64)).to(device)
    traj, dens = golden_angle_radial(nfe, spf, T)
    traj, dens = torch.from_numpy(traj).to(device), torch.from_numpy(dens).to(device)
    op = av.RadialOperator(W, H, C, T, traj, dens, spf, kernel_width, sector_width, osf)
    k = op.backward(x, b1)
    sd = noise_rel * float(k.abs().max())
    g = torch.Generator(device=device)
    g.manual_seed(spec["seed"])
    k += (sd / np.sqrt(2.0)) * torch.complex(torch.randn(k.shape, generator=g, device=device),
                                            torch.randn(k.shape, generator=g, device=device))
    del op
    return dict(kdata=k, traj=traj, dens=dens, b1=b1, x0=torch.zeros((T, H, W), dtype=torch.complex64,
                                                                     device=device), n_fe=nfe, spokes=spf,
                kernel_width=kernel_width, sector_width=sector_width, osf=osf)


def serving_stream(seed=4, n=2000, rate=20.0):
    """Request specs of the serving configuration with Poisson arrival times
    (seconds from the start) at the given rate."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for i in range(n):
        method = ("TV", "TGV2", "ICTGV2")[int(rng.choice(3, p=[0.5, 0.3, 0.2]))]
        if rng.random() < 0.7:
            m = int(rng.choice(MATRICES))
            spec = dict(kind="cartesian", W=m, H=m, T=int(rng.integers(8, 49)), C=int(rng.integers(4, 33)),
                        R=int(rng.integers(6, 17)))
        else:
            spec = dict(kind="radial", W=128, H=128, T=int(rng.integers(20, 61)), C=12,
                        spokes=int(rng.integers(13, 35)), n_fe=256)
        spec.update(method=method, arrival=float(t[i]), seed=int(rng.integers(1 << 31)))
        out.append(spec)
    return out


def nudft_gpu(u, traj_f):
    """Exact non-uniform DFT in float64 on the GPU:
    X[..., s] = sum_{y,x} u[..., y, x] exp(-2 pi i (kx_s px + ky_s py)),
    p = index - floor(extent / 2); u (..., H, W) complex128, traj_f (2, S)."""
    import torch
    H, W = u.shape[-2:]
    dev = u.device
    kx = traj_f[0].to(dev, torch.float64)
    ky = traj_f[1].to(dev, torch.float64)
    px = torch.arange(W, device=dev, dtype=torch.float64) - W // 2
    py = torch.arange(H, device=dev, dtype=torch.float64) - H // 2
    ex = torch.exp(-2j * np.pi * torch.outer(px, kx))   # (W, S)
    ey = torch.exp(-2j * np.pi * torch.outer(py, ky))   # (H, S)
    return ((u @ ex) * ey).sum(-2)


def radial_128_gpu(seed=2, H=128, W=128, T=40, C=12, n_fe=256, spokes=21, noise_rel=2e-3, device="cuda"):
    """The radial configuration: returns CUDA tensors kdata (T, C, S)
    sqrt(w)-weighted, traj (T, 2, S), dens (T, S) and the phantom."""
    import torch
    rng = np.random.default_rng(seed)
    x = torch.from_numpy(phantom_cine(H, W, T, rng, period=30)).to(device)
    b1 = torch.from_numpy(coil_maps(H, W, C, rng)).to(device)
    traj, dens = golden_angle_radial(n_fe, spokes, T)
    traj_d, dens_d = torch.from_numpy(traj).to(device), torch.from_numpy(dens).to(device)
    S = traj.shape[2]
    k = torch.empty((T, C, S), dtype=torch.complex128, device=device)
    for t in range(T):
        k[t] = nudft_gpu(b1 * x[t], traj_d[t]) / np.sqrt(W * H)
    sd = noise_rel * float(k.abs().max())
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    k += (sd / np.sqrt(2.0)) * torch.complex(torch.randn(k.shape, generator=g, device=device, dtype=torch.float64),
                                            torch.randn(k.shape, generator=g, device=device, dtype=torch.float64))
    k *= torch.sqrt(dens_d.double())[:, None, :]
    return dict(kdata=k.to(torch.complex64).contiguous(), traj=traj_d, dens=dens_d, truth=x.to(torch.complex64),
                n_fe=n_fe, spokes=spokes)


# ---------------------------------------------------------------------------
# problems with float64-oracle fixtures (numpy only, reproducible bit for bit)
# ---------------------------------------------------------------------------

# The cine benchmark's solver parameters: the reference's default configuration
# file's [ictgv2] section, 1000 iterations, no gap evaluation.
CINE_192_PARAMS = dict(maxIt=1000, stopPDGap=0.0, sigma=0.3333, tau=0.3333, sigmaTauRatio=1.0,
                       timeSpaceWeight=4.0, timeSpaceWeight2=0.5, alpha=0.5, alpha0=1.41421356, alpha1=1.0,
                       **{"lambda": 6.0})
BATCHED_ITERS = 800
TV_ELLIPSES_ITERS = 500
RADIAL_ITERS = 500


def tv_ellipses_128_problem(seed=0):
    """``tv_ellipses_128`` with its initial image (the coil-combined
    zero-filled time average)."""
    prob = tv_ellipses_128(seed)
    prob["u0"] = time_average_u0(prob["kdata"], prob["mask"], prob["b1"])
    return prob


def cine_192_problem(seed=1):
    """``cine_192`` with the initial image the benchmark starts from (the
    coil-combined zero-filled time average, replicated over the frames)."""
    prob = cine_192(seed)
    prob["u0"] = time_average_u0(prob["kdata"], prob["mask"], prob["b1"])
    return prob


def cine_instance(spec, noise_rel=1e-3):
    """A batched instance generated on the host (numpy arrays: kdata
    (T,C,H,W) masked, mask, b1, u0 (H,W)): the problems the float64 oracle
    fixtures hold.  Same construction as ``cine_instance_gpu``; the noise
    comes from the spec's numpy generator."""
    H, W, T, C = spec["H"], spec["W"], spec["T"], spec["C"]
    rng = np.random.default_rng(spec["seed"])
    x = phantom_cine(H, W, T, rng, period=30)
    b1 = coil_maps(H, W, C, rng)
    mask = mask_variable_density(H, W, T, R=spec["R"], rng=rng)
    k = simulate(x, b1, mask, rng, noise_rel).astype(np.complex64)
    b1 = b1.astype(np.complex64)
    return dict(kdata=k, mask=mask, b1=b1, u0=time_average_u0(k, mask, b1), truth=x.astype(np.complex64))


def oracle_batched_indices(seed=3, n=64):
    """Instances of the batched set with oracle fixtures: size ranks 0, 16,
    32 and 48 of 64 (by W H T C, ties by index), one per quartile below the
    largest."""
    specs = batched_specs(seed, n)
    order = sorted(range(n), key=lambda i: (specs[i]["W"] * specs[i]["H"] * specs[i]["T"] * specs[i]["C"], i))
    return [order[r] for r in (0, n // 4, n // 2, 3 * n // 4)]


def nudft(u, traj_f):
    """Exact non-uniform DFT in float64 (numpy):
    X[..., s] = sum_{y,x} u[..., y, x] exp(-2 pi i (kx_s px + ky_s py)),
    p = index - floor(extent / 2); u (..., H, W), traj_f (2, S)."""
    H, W = u.shape[-2:]
    kx = traj_f[0].astype(np.float64)
    ky = traj_f[1].astype(np.float64)
    px = np.arange(W, dtype=np.float64) - W // 2
    py = np.arange(H, dtype=np.float64) - H // 2
    ex = np.exp(-2j * np.pi * np.outer(px, kx))   # (W, S)
    ey = np.exp(-2j * np.pi * np.outer(py, ky))   # (H, S)
    return ((u @ ex) * ey).sum(-2)


def radial_128(seed=2, H=128, W=128, T=40, C=12, n_fe=256, spokes=21, noise_rel=2e-3):
    """The radial configuration generated on the host (numpy): kdata (T, C, S)
    complex64, sqrt(w)-weighted as the CLI weights it (main.cpp:546-570),
    traj (T, 2, S) and dens (T, S) float32, the phantom (T, H, W); k-space by
    the exact float64 NUDFT, complex Gaussian noise at noise_rel of max |k|."""
    rng = np.random.default_rng(seed)
    x = phantom_cine(H, W, T, rng, period=30)
    b1 = coil_maps(H, W, C, rng)
    traj, dens = golden_angle_radial(n_fe, spokes, T)
    S = traj.shape[2]
    k = np.empty((T, C, S), dtype=np.complex128)
    for t in range(T):
        k[t] = nudft(b1 * x[t], traj[t]) / np.sqrt(W * H)
    sd = noise_rel * np.max(np.abs(k))
    k += (sd / np.sqrt(2.0)) * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape))
    k *= np.sqrt(dens.astype(np.float64))[:, None, :]
    return dict(kdata=k.astype(np.complex64), traj=traj, dens=dens, truth=x.astype(np.complex64), n_fe=n_fe,
                spokes=spokes, b1_true=b1.astype(np.complex64))
