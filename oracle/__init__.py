"""Float64 CPU oracle for the AVIONIC primal-dual reconstruction path.

TEST INFRASTRUCTURE ONLY.  This package restates, in numpy float64, the
arithmetic of the reference's TV / TGV2 / ICTGV2 Chambolle-Pock loops, its
finite-difference stencils, norm-ball projections, step-size rule, primal-dual
gap and Cartesian multi-coil operator.  It is the checker that the CUDA path
is compared against: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it.  The product library
(``avionic_b200`` / ``libavionic_core.so``) never routes through it.

Pinning: every function here is checked against the known-answer values that
the reference's own gtest suite holds (``CUDA/test/derivatives.cc``,
``tv.cc``, ``tgv2.cc``, ``ictgv2.cc``, ``fft.cc``, ``utils.cc``,
``cartesian_operator.cc``), transcribed with file:line citations in
``tests/golden/reference_kats.json``.  The reference itself (C++ on top of the
unvendored AGILE and gpuNUFFT libraries, and MATLAB) cannot be built or run in
this environment, so those KATs are the pin.

Array conventions (the reference's linear layouts, as numpy shapes):
  image       (T, H, W)        index x + W*(y + H*t)
  k-space     (T, C, H, W)     index x + W*(y + H*(c + C*t))
  coil maps   (C, H, W)        index x + W*(y + H*c)
  mask        (T, H, W)        float, index x + W*(y + H*t)
"""

from . import stencils, cartesian, solvers, binfmt  # noqa: F401
