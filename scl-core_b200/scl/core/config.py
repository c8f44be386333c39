"""Precision / library-variant selection (mirrors python/scl/core/config.py).

scl-core's wrapper always picks int64 indices; here the index width follows
the data when it is given (all four variants are built), and ``set_precision``
sets the default as in the reference.
"""
from __future__ import annotations

import ctypes
from enum import Enum
from typing import Optional, Tuple, Union

import numpy as np

from .._bindings._loader import Library, get_library as _get_library


class RealType(Enum):
    FLOAT32 = "f32"
    FLOAT64 = "f64"

    @property
    def numpy_dtype(self):
        return np.float32 if self == RealType.FLOAT32 else np.float64

    @property
    def ctypes_type(self):
        return ctypes.c_float if self == RealType.FLOAT32 else ctypes.c_double


class IndexType(Enum):
    INT32 = "i32"
    INT64 = "i64"

    @property
    def numpy_dtype(self):
        return np.int32 if self == IndexType.INT32 else np.int64

    @property
    def ctypes_type(self):
        return ctypes.c_int32 if self == IndexType.INT32 else ctypes.c_int64


_REAL_ALIASES = {"float32": RealType.FLOAT32, "f32": RealType.FLOAT32, "float64": RealType.FLOAT64,
                 "f64": RealType.FLOAT64}
_INDEX_ALIASES = {"int32": IndexType.INT32, "i32": IndexType.INT32, "int64": IndexType.INT64, "i64": IndexType.INT64}


class _Config:
    def __init__(self):
        self.default_real = RealType.FLOAT64
        self.default_index = IndexType.INT64

    @property
    def default_variant(self) -> str:
        return f"{self.default_real.value}_{self.default_index.value}"


_config = _Config()


def get_config() -> _Config:
    return _config


def set_precision(real: Optional[Union[RealType, str]] = None, index: Optional[Union[IndexType, str]] = None) -> None:
    if real is not None:
        _config.default_real = real if isinstance(real, RealType) else _REAL_ALIASES[str(real)]
    if index is not None:
        _config.default_index = index if isinstance(index, IndexType) else _INDEX_ALIASES[str(index)]


def get_precision() -> Tuple[RealType, IndexType]:
    return _config.default_real, _config.default_index


def get_library(variant: Optional[str] = None) -> Library:
    return _get_library(variant or _config.default_variant)


def infer_variant(data: Optional[np.ndarray] = None, index: Optional[np.ndarray] = None) -> str:
    real = _config.default_real
    if data is not None:
        real = RealType.FLOAT32 if data.dtype == np.float32 else RealType.FLOAT64
    idx = _config.default_index
    if index is not None:
        idx = IndexType.INT32 if index.dtype == np.int32 else IndexType.INT64
    return f"{real.value}_{idx.value}"


def _infer_library(data=None, indices=None) -> Library:
    return get_library(infer_variant(data, indices))
