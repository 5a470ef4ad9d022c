"""Data normalisation of the CLI's -o switch, float64 (test infrastructure).

Restates RawDataPreparation::NormalizeData (CUDA/src/raw_data_preparation.cpp
:340-378) for binary input: NormalizeCartData (:821-844) with the centred
Cartesian time average, NormalizeNonCartData (:742-786) with the radial one
(kernel width 3, sector width 8, osf 2), and FindNormalizationFactor
(:661-686) with utils::Median (CUDA/src/utils.cpp:1442-1462).
"""

import numpy as np

from .coils import time_averaged_radial, time_averaged_reconstruction


def find_normalization_factor(values):
    """The first largest value, then every later value (scan order) that is
    >= 0.9 of it; the median of those (mean of the two middle values for an
    even count).  Values before the first maximum are not considered."""
    v = np.asarray(values, dtype=np.float64).ravel()
    i = int(np.argmax(v))
    big = np.concatenate([[v[i]], v[i + 1:][v[i + 1:] >= 0.9 * v[i]]])
    big.sort()
    ind = int(big.size * 0.5)
    if big.size % 2 == 0:
        return 0.5 * (big[ind] + big[ind - 1])
    return big[ind]


def normalization_factor(kdata, mask=None, traj=None, dens=None, W=None, H=None):
    """Cartesian (mask given; kdata (T,C,H,W)): 255 / m of the centred time
    average's |u|.  Radial (traj, dens, W, H given; kdata (T,C,S)):
    255 T / m of sqrt(sum_c |crec_c|^2).  Returns the factor; the CLI scales
    its k-space by it."""
    if traj is None:
        u, _ = time_averaged_reconstruction(kdata, mask, centered=True, apply_phase=False)
        return 255.0 / find_normalization_factor(np.abs(u))
    u, _ = time_averaged_radial(kdata, traj, dens, W, H, apply_phase=False)
    return 255.0 * kdata.shape[0] / find_normalization_factor(np.abs(u))
