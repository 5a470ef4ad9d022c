"""Non-Cartesian (radial) multi-coil operator, float64 (test infrastructure).

The reference's radial operator (CUDA/src/noncartesian_operator.cpp:3-195)
delegates to gpuNUFFT (andyschwarzl/gpuNUFFT, branch deapo-scaling, no pinned
commit, not in the tree).  Its MATLAB twin (matlab/backward_opt_noncart.m:12-21,
matlab/forward_opt_noncart.m:9-18) defines the operator as
    K_f x   = sqrt(w_f) * NUFFT_f(b1_c * x_f) / sqrt(H W)            (image -> k)
    K_f^H z = sum_c conj(b1_c) * NUFFT_f^H(sqrt(w_f) * z_{f,c}) / sqrt(H W)
with NUFFT the non-uniform DFT  X(k) = sum_n u[n] exp(-2 pi i k . (n - N/2)),
k in [-0.5, 0.5) cycles/pixel per axis.  gpuNUFFT's exact kernel, scaling and
sector layout cannot be reproduced without its source, so radial parity is
*unpinned* against the reference; this module fixes one gridding definition
that the CUDA path implements identically, and checks it against the exact
NUDFT (its approximation error) and for adjointness:

* kernel: Kaiser-Bessel with the Beatty et al. (2005) shape parameter
  beta = pi sqrt((J/osf)^2 (osf - 1/2)^2 - 0.8), tapered to reach zero at the
  window edge: w(u) = (I0(beta sqrt(1 - (2u/J)^2)) - 1) / (I0(beta) - 1),
  |u| < J/2 (grid units), J = kernelWidth;
* grid: G_d = 2 ceil(osf d / 2) per axis; pixel n sits at position
  p = n - floor(d/2) and grid index p mod G_d; forward transform
  V[g] = sum_m v[m] exp(-2 pi i g m / G_d) (unnormalised);
* deapodisation: divide by psi(p) = int w(t) cos(2 pi t p / G_d) dt per axis
  (64-point Gauss-Legendre), which makes sum_g w(kG - g) V[g] an unbiased
  approximation of the NUDFT;
* interpolation at kappa = k G_d over the integers g with |kappa - g| < J/2.

Data layout follows the reference: trajectory per frame [kx(S) | ky(S)]
(matlab/avionic_matlab_gpu.m:183-189), k-space [frame][coil][sample]
(noncartesian_operator.cpp:117-121), density [frame][sample].
"""

import numpy as np


def _smooth13(n):
    for p in (2, 3, 5, 7, 11, 13):
        while n % p == 0:
            n //= p
    return n == 1


def grid_size(d, osf):
    """Smallest even size >= osf d whose prime factors are <= 13."""
    n = int(2 * np.ceil(osf * d / 2.0))
    while not _smooth13(n):
        n += 2
    return n


def kb_beta(J, osf):
    return np.pi * np.sqrt((J / osf) ** 2 * (osf - 0.5) ** 2 - 0.8)


def kb(u, J, beta):
    u = np.asarray(u, dtype=np.float64)
    a = 1.0 - (2.0 * u / J) ** 2
    out = np.zeros_like(u)
    inside = np.abs(u) < J / 2.0
    out[inside] = (np.i0(beta * np.sqrt(a[inside])) - 1.0) / (np.i0(beta) - 1.0)
    return out


def deapodization(d, G, J, beta, nodes=64):
    """psi(p) for p = n - floor(d/2), n = 0..d-1."""
    xg, wg = np.polynomial.legendre.leggauss(nodes)
    t = xg * (J / 2.0)
    wt = wg * (J / 2.0) * kb(t, J, beta)
    p = np.arange(d) - d // 2
    return np.array([np.sum(wt * np.cos(2 * np.pi * t * pp / G)) for pp in p])


def sector_map(traj, G, sector_width):
    """Sector layout of the samples, in float32 arithmetic as the device
    library computes it: grid position g = k G (float32), wrapped into [0, G)
    by adding G when negative; sector = clamp(floor(g / sw), 0, nsec - 1) per
    axis; sector index sy * nsx + sx.  Returns (order [T, S]: sample indices
    sorted by sector, stable; start [T, nsx*nsy + 1]: offsets into order)."""
    Gy, Gx = G
    sw = np.float32(sector_width)
    nsx = int(np.ceil(Gx / sector_width))
    nsy = int(np.ceil(Gy / sector_width))
    gx = traj[:, 0, :].astype(np.float32) * np.float32(Gx)
    gy = traj[:, 1, :].astype(np.float32) * np.float32(Gy)
    gx = np.where(gx < 0, gx + np.float32(Gx), gx).astype(np.float32)
    gy = np.where(gy < 0, gy + np.float32(Gy), gy).astype(np.float32)
    sx = np.clip(np.floor(gx / sw).astype(np.int64), 0, nsx - 1)
    sy = np.clip(np.floor(gy / sw).astype(np.int64), 0, nsy - 1)
    sec = sy * nsx + sx
    order = np.argsort(sec, axis=1, kind="stable")
    start = np.zeros((traj.shape[0], nsx * nsy + 1), dtype=np.int64)
    for f in range(traj.shape[0]):
        start[f, 1:] = np.cumsum(np.bincount(sec[f], minlength=nsx * nsy))
    return order, start


class RadialOperator:
    """Oracle twin of the radial operator (see module docstring)."""

    def __init__(self, width, height, coils, frames, traj, dens, kernel_width=3.0, sector_width=8.0, osf=2.0):
        self.W, self.H, self.C, self.T = width, height, coils, frames
        self.traj = np.asarray(traj, dtype=np.float64)     # (T, 2, S)
        self.dens = np.asarray(dens, dtype=np.float64)     # (T, S)
        self.S = self.traj.shape[2]
        self.J = float(kernel_width)
        self.osf = float(osf)
        self.sw = float(sector_width)
        self.Gx, self.Gy = grid_size(width, osf), grid_size(height, osf)
        self.beta = kb_beta(self.J, self.osf)
        self.psi_x = deapodization(width, self.Gx, self.J, self.beta)
        self.psi_y = deapodization(height, self.Gy, self.J, self.beta)
        self.sqrt_w = np.sqrt(self.dens)
        self.norm = 1.0 / np.sqrt(width * height)
        self._prep()

    def _prep(self):
        """Interpolation stencils: per sample the grid indices and weights."""
        J, nwin = self.J, int(np.ceil(self.J)) + 1
        self.ix, self.iy, self.wx, self.wy = [], [], [], []
        for f in range(self.T):
            kap_x = self.traj[f, 0] * self.Gx
            kap_y = self.traj[f, 1] * self.Gy
            g0x = np.floor(kap_x - J / 2.0).astype(np.int64)
            g0y = np.floor(kap_y - J / 2.0).astype(np.int64)
            offs = np.arange(nwin)
            gx = g0x[:, None] + offs[None, :]
            gy = g0y[:, None] + offs[None, :]
            self.wx.append(kb(kap_x[:, None] - gx, J, self.beta))
            self.wy.append(kb(kap_y[:, None] - gy, J, self.beta))
            self.ix.append(np.mod(gx, self.Gx))
            self.iy.append(np.mod(gy, self.Gy))

    def _pad(self, u):
        """image (H, W) / deapodisation -> grid (Gy, Gx)."""
        v = np.zeros((self.Gy, self.Gx), dtype=np.complex128)
        py = np.mod(np.arange(self.H) - self.H // 2, self.Gy)
        px = np.mod(np.arange(self.W) - self.W // 2, self.Gx)
        v[np.ix_(py, px)] = u / (self.psi_y[:, None] * self.psi_x[None, :])
        return v

    def _crop(self, v):
        py = np.mod(np.arange(self.H) - self.H // 2, self.Gy)
        px = np.mod(np.arange(self.W) - self.W // 2, self.Gx)
        return v[np.ix_(py, px)] / (self.psi_y[:, None] * self.psi_x[None, :])

    def _interp(self, V, f):
        vals = V[self.iy[f][:, :, None], self.ix[f][:, None, :]]
        w = self.wy[f][:, :, None] * self.wx[f][:, None, :]
        return np.sum(vals * w, axis=(1, 2))

    def _spread(self, z, f):
        V = np.zeros((self.Gy, self.Gx), dtype=np.complex128)
        w = self.wy[f][:, :, None] * self.wx[f][:, None, :] * z[:, None, None]
        iy = np.broadcast_to(self.iy[f][:, :, None], w.shape)
        ix = np.broadcast_to(self.ix[f][:, None, :], w.shape)
        np.add.at(V, (iy.ravel(), ix.ravel()), w.ravel())
        return V

    def backward(self, x, b1):
        """image (T,H,W) -> samples (T,C,S) (BackwardOperation)."""
        out = np.zeros((self.T, self.C, self.S), dtype=np.complex128)
        for f in range(self.T):
            for c in range(self.C):
                V = np.fft.fft2(self._pad(b1[c] * x[f]))
                out[f, c] = self._interp(V, f) * self.sqrt_w[f] * self.norm
        return out

    def forward(self, z, b1, inplace_mask=True):
        """samples (T,C,S) -> image (T,H,W) (ForwardOperation)."""
        out = np.zeros((self.T, self.H, self.W), dtype=np.complex128)
        for f in range(self.T):
            for c in range(self.C):
                V = self._spread(z[f, c] * self.sqrt_w[f] * self.norm, f)
                # adjoint of the unnormalised forward FFT: G * ifft2
                img = self._crop(np.fft.ifft2(V) * (self.Gx * self.Gy))
                out[f] += np.conj(b1[c]) * img
        return out

    def adapt_lambda(self, k, d, spokes_per_frame):
        """noncartesian_operator.cpp:88-95: lambda = W / (spf pi / 2) k + d."""
        return self.W / (spokes_per_frame * np.pi / 2.0) * k + d


def nudft(u, traj_f):
    """Exact X(k) = sum_n u[n] exp(-2 pi i (kx px + ky py)), p = n - floor(d/2)."""
    H, W = u.shape
    py = np.arange(H) - H // 2
    px = np.arange(W) - W // 2
    ex = np.exp(-2j * np.pi * np.outer(traj_f[0], px))   # (S, W)
    ey = np.exp(-2j * np.pi * np.outer(traj_f[1], py))   # (S, H)
    return np.einsum("sh,hw,sw->s", ey, u, ex)


def golden_angle_radial(n_ro, spokes_per_frame, frames, angle_deg=111.246117975):
    """Golden-angle radial trajectory (T, 2, S) in [-0.5, 0.5) and a ramp
    density (normalised to max 1), readout of n_ro samples."""
    r = (np.arange(n_ro) - n_ro / 2.0) / n_ro
    traj = np.zeros((frames, 2, n_ro * spokes_per_frame))
    dens = np.zeros((frames, n_ro * spokes_per_frame))
    a = 0
    for f in range(frames):
        for s in range(spokes_per_frame):
            th = np.deg2rad(angle_deg) * a
            a += 1
            sl = slice(s * n_ro, (s + 1) * n_ro)
            traj[f, 0, sl] = r * np.cos(th)
            traj[f, 1, sl] = r * np.sin(th)
            dens[f, sl] = np.abs(r) + 0.5 / n_ro
    dens /= dens.max()
    return traj, dens
