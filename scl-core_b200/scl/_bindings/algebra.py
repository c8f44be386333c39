"""Bindings of include/scl_algebra.h (scl-core algebra.h:121-140)."""
from ._loader import Error, Index, Ptr, Real, SparseHandle, register


@register
def scl_algebra_spmm(A: SparseHandle, X: Ptr[Real], n_cols: Index, Y: Ptr[Real], alpha: Real, beta: Real) -> Error: ...
