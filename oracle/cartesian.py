"""Cartesian multi-coil MR operator (float64).

Test infrastructure (see ``oracle/__init__``).  Restates
``CUDA/src/cartesian_operator.cpp`` of the reference:

* ``backward`` (image -> k-space, cartesian_operator.cpp:122-160):
  k[t, c] = mask[t] * F(b1[c] * x[t]);
* ``forward`` (k-space -> image, cartesian_operator.cpp:65-111):
  x[t] = sum_c conj(b1[c]) * F^-1(mask[t] * k[t, c]).  Like the reference it
  multiplies its k-space input by the mask in place (:83-88);
* ``adapt_lambda`` (:47-62).

F is the unitary 2D DFT over (H, W) with the e^{+2 pi i k n / N} kernel for
image -> k-space and e^{-2 pi i k n / N} for k-space -> image.  The
reference's FFT tests (CUDA/test/fft.cc:58-64) pin only magnitudes; the sign
is pinned by the 500-iteration solver goldens (CUDA/test/tv.cc:482-485,
tgv2.cc:544-549, ictgv2.cc:674-679), which the opposite sign misses by up to
3e-3 (tolerance 1e-3).  It is also the MATLAB twin's convention
(matlab/backward_opt.m:12 uses ifft2 for image -> k-space).  ``centered=True``
applies fftshift(F(ifftshift(.))) per slice, the AGILE ``CenteredForward``
used by the reference's default-constructed operator (the CLI uses the
uncentred form, main.cpp:755-756).
"""

import numpy as np

# When set (an int), the 2D transforms run through scipy.fft with that many
# threads; used only to time the oracle on all host cores.
FFT_WORKERS = None


def _fft2(a):
    if FFT_WORKERS:
        import scipy.fft as sf
        return sf.fft2(a, norm="ortho", workers=FFT_WORKERS)
    return np.fft.fft2(a, norm="ortho")


def _ifft2(a):
    if FFT_WORKERS:
        import scipy.fft as sf
        return sf.ifft2(a, norm="ortho", workers=FFT_WORKERS)
    return np.fft.ifft2(a, norm="ortho")


def fft2u(a, centered=False):
    """Unitary image -> k-space transform (e^{+2 pi i} kernel)."""
    if centered:
        a = np.fft.ifftshift(a, axes=(-2, -1))
    r = _ifft2(a)
    if centered:
        r = np.fft.fftshift(r, axes=(-2, -1))
    return r


def ifft2u(a, centered=False):
    """Unitary k-space -> image transform (e^{-2 pi i} kernel)."""
    if centered:
        a = np.fft.ifftshift(a, axes=(-2, -1))
    r = _fft2(a)
    if centered:
        r = np.fft.fftshift(r, axes=(-2, -1))
    return r


class CartesianOperator:
    """Oracle twin of ``CartesianOperator`` (cartesian_operator.h:22-125).

    ``mask`` is None for the reference's empty-mask constructors
    (cartesian_operator.cpp:19-34) or a float array (T, H, W)."""

    def __init__(self, width, height, coils, frames, mask=None, centered=True):
        self.W, self.H, self.C, self.T = width, height, coils, frames
        self.mask = None if mask is None else np.asarray(mask, dtype=np.float64)
        self.centered = centered

    def backward(self, x, b1):
        """image (T,H,W) -> k-space (T,C,H,W)."""
        k = fft2u(b1[None, :, :, :] * x[:, None, :, :], self.centered)
        if self.mask is not None:
            k = k * self.mask[:, None, :, :]
        return k

    def forward(self, z, b1, inplace_mask=True):
        """k-space (T,C,H,W) -> image (T,H,W).  When ``inplace_mask`` the
        masked k-space is written back into ``z`` as the reference does."""
        if self.mask is not None:
            zm = z * self.mask[:, None, :, :]
            if inplace_mask:
                z[...] = zm
        else:
            zm = z
        img = ifft2u(zm, self.centered)
        return np.sum(np.conj(b1)[None, :, :, :] * img, axis=1)

    def adapt_lambda(self, k, d):
        """lambda = k * W*H*T/||mask||^2 + d (cartesian_operator.cpp:47-62)."""
        subfac = float(self.W * self.H * self.T)
        if self.mask is not None:
            subfac /= float(np.sum(self.mask.astype(np.float64) ** 2))
        else:
            subfac /= float(self.W * self.H * self.T)
        return subfac * k + d
