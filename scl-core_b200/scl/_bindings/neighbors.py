"""Bindings of include/scl_neighbors.h (scl-core neighbors/neighbors.h:18-41)."""
from ._loader import Error, Index, Ptr, Real, Size, SparseHandle, register


@register
def scl_neighbors_compute_norms(matrix: SparseHandle, norms_sq: Ptr[Real]) -> Error: ...
@register
def scl_knn(matrix: SparseHandle, norms_sq: Ptr[Real], n_samples: Size, k: Size, out_indices: Ptr[Index],
            out_distances: Ptr[Real]) -> Error: ...
@register
def scl_knn_simple(matrix: SparseHandle, n_samples: Size, k: Size, out_indices: Ptr[Index],
                   out_distances: Ptr[Real]) -> Error: ...
