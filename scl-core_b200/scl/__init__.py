"""B200 drop-in for scl-core's graph-diffusion path.

Mirrors scl-core's ``python/scl`` package for this path: ``CsrMatrix`` handles,
``set_precision`` variant selection, ``check_error``/``SCLError``, and the
``scl_diffusion_*`` calls in :mod:`scl.diffusion`. Device-resident graphs for
torch callers live in :mod:`scl.gpu`.
"""
from . import _bindings  # noqa: F401  (binds every registered C function)
from .core import (BlockStrategy, CsrMatrix, IndexType, RealType, SCLError, check_error, get_library,  # noqa: F401
                   get_precision, set_precision)
from . import algebra, diffusion, gpu, impute, neighbors, synthetic  # noqa: F401

__version__ = "1.0.0"
