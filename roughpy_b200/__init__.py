"""roughpy_b200: RoughPy's dense truncated tensor-algebra hot path on NVIDIA B200.

* ``roughpy_b200.compute``  -- drop-in for ``roughpy.compute`` (ft_fma, ft_mul,
  ft_exp, ft_log, ft_fmexp, antipode, Lie maps, ...), GPU kernels throughout.
* ``roughpy_b200.signatures`` -- batched path signatures (Chen products).
* ``roughpy_b200.streams`` -- LieIncrementStream-compatible streams with dyadic
  caching and batched interval queries.

All computation goes through ``librpyb.so`` (C ABI in ``include/rpyb.h``).
"""
from . import _lib  # noqa: F401  (fails loudly if the library is not built)

__version__ = "0.1.0"


def version() -> str:
    return _lib.version()
