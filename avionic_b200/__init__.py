"""Python host mirror of the AVIONIC B200 reconstruction core.

The product is ``libavionic_core.so`` (CUDA, sm_100a) behind the C ABI in
``include/avionic.h``; ``avionic_b200.api`` binds it with ctypes and mirrors
the reference's interface for the reconstruction path (``CartesianOperator``,
``RadialOperator``, the ``TV``/``TGV2``/``ICTGV2`` solvers, ``utils``
stencils, the batch engine).  Every public name of ``api`` is available here:
the first such access loads the library, and fails loudly when it is missing
(there is no CPU fallback).  ``avionic_b200.synth`` (seeded numpy problem
generators) imports without loading the library.
"""

_SUBMODULES = ("api", "synth", "_abi")


def __getattr__(name):
    if name in _SUBMODULES or name.startswith("__"):
        raise AttributeError(name)
    from . import api
    return getattr(api, name)


def __dir__():
    from . import api
    return sorted(set(globals()) | {n for n in dir(api) if not n.startswith("_")})
