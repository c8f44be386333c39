"""Bindings of include/scl_impute.h (scl-core impute/impute.h:15-58)."""
from ._loader import Error, Index, Ptr, Real, SparseHandle, register


@register
def scl_impute_knn(matrix: SparseHandle, knn_indices: Ptr[Index], knn_distances: Ptr[Real], n_cells: Index,
                   n_genes: Index, k_neighbors: Index, X_imputed: Ptr[Real], bandwidth: Real,
                   threshold: Real) -> Error: ...
@register
def scl_impute_knn_weighted(matrix: SparseHandle, knn_indices: Ptr[Index], knn_distances: Ptr[Real], n_cells: Index,
                            n_genes: Index, k_neighbors: Index, X_imputed: Ptr[Real], bandwidth: Real,
                            threshold: Real) -> Error: ...
@register
def scl_impute_diffusion(matrix: SparseHandle, transition_matrix: SparseHandle, n_cells: Index, n_genes: Index,
                         n_steps: Index, X_imputed: Ptr[Real]) -> Error: ...
@register
def scl_impute_magic(matrix: SparseHandle, affinity_matrix: SparseHandle, n_cells: Index, n_genes: Index, t: Index,
                     X_imputed: Ptr[Real]) -> Error: ...
