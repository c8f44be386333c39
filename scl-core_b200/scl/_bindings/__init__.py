"""ctypes bindings (hand-written in the style scl-core's codegen emits)."""
from . import algebra, core, diffusion, gpu, impute, neighbors, sparse  # noqa: F401  (register all functions)
from ._loader import Library, VARIANTS, get_library  # noqa: F401
