"""ctypes loader for the B200 diffusion libraries.

Mirrors the loader that scl-core generates (codegen/cli.py:236-660): functions
are declared once with ``@register`` and type-hint markers, and each
``Library(variant)`` binds them against ``libscl_<variant>.so`` found in
``scl/libs``, the working directory or ``$SCL_LIB_DIR``.
"""
from __future__ import annotations

import ctypes
import inspect
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Dict, Optional, get_type_hints


# ---- type markers (resolved per variant) -----------------------------------
class Real: ...
class Index: ...
class Size: ...
class Error: ...
class Bool: ...
class Int: ...
class Int64: ...
class Double: ...
class SparseHandle: ...
class GpuGraphHandle: ...
class VoidPtr: ...
class CharPtr: ...


class Ptr:
    def __class_getitem__(cls, item):
        return type(f"Ptr[{getattr(item, '__name__', item)}]", (), {"_pointee": item})


@dataclass(frozen=True)
class VariantInfo:
    real_type: str
    index_type: str
    ctypes_real: type
    ctypes_index: type


VARIANTS: Dict[str, VariantInfo] = {
    "f32_i32": VariantInfo("float32", "int32", ctypes.c_float, ctypes.c_int32),
    "f32_i64": VariantInfo("float32", "int64", ctypes.c_float, ctypes.c_int64),
    "f64_i32": VariantInfo("float64", "int32", ctypes.c_double, ctypes.c_int32),
    "f64_i64": VariantInfo("float64", "int64", ctypes.c_double, ctypes.c_int64),
}
DEFAULT_VARIANT = "f64_i64"


@dataclass
class FunctionSpec:
    name: str
    func: Callable


_FUNCTION_REGISTRY: Dict[str, FunctionSpec] = {}


def register(func: Callable) -> Callable:
    _FUNCTION_REGISTRY[func.__name__] = FunctionSpec(func.__name__, func)
    return func


def get_registered_functions():
    return list(_FUNCTION_REGISTRY)


def _build_type_map(v: VariantInfo) -> dict:
    return {
        Real: v.ctypes_real, Index: v.ctypes_index, Size: ctypes.c_size_t, Error: ctypes.c_int32,
        Bool: ctypes.c_int, Int: ctypes.c_int, Int64: ctypes.c_int64, Double: ctypes.c_double,
        SparseHandle: ctypes.c_void_p, GpuGraphHandle: ctypes.c_void_p, VoidPtr: ctypes.c_void_p,
        CharPtr: ctypes.c_char_p, None: None, type(None): None,
    }


def _resolve_type(hint, tmap):
    if hint in tmap:
        return tmap[hint]
    pointee = getattr(hint, "_pointee", None)
    if pointee is not None:
        base = _resolve_type(pointee, tmap)
        return ctypes.POINTER(base) if base is not None else ctypes.c_void_p
    return ctypes.c_void_p


LIBS_DIR = Path(__file__).resolve().parent.parent / "libs"


def _lib_name(variant: str) -> str:
    return f"libscl_{variant}.so"


def find_library(variant: str) -> Optional[Path]:
    paths = [LIBS_DIR, Path.cwd()]
    env = os.environ.get("SCL_LIB_DIR")
    if env:
        paths.append(Path(env))
    for base in paths:
        p = base / _lib_name(variant)
        if p.exists():
            return p
    return None


class Library:
    """One library variant with every registered function bound on load."""

    def __init__(self, variant: str, lazy: bool = True):
        if variant not in VARIANTS:
            raise ValueError(f"Unknown variant '{variant}'. Available: {list(VARIANTS)}")
        self._variant = variant
        self._info = VARIANTS[variant]
        self._tmap = _build_type_map(self._info)
        self._native: Optional[ctypes.CDLL] = None
        self._functions: Dict[str, Callable] = {}
        if not lazy:
            self._ensure_loaded()

    variant = property(lambda self: self._variant)
    real_type = property(lambda self: self._info.ctypes_real)
    index_type = property(lambda self: self._info.ctypes_index)
    is_loaded = property(lambda self: self._native is not None)

    @property
    def path(self) -> Optional[Path]:
        return find_library(self._variant)

    def _ensure_loaded(self):
        if self._native is not None:
            return
        p = find_library(self._variant)
        if p is None:
            raise RuntimeError(f"Cannot find library '{_lib_name(self._variant)}'. "
                               f"Build it with: python scl-core_b200/build.py")
        self._native = ctypes.CDLL(str(p))
        for name, spec in _FUNCTION_REGISTRY.items():
            try:
                self._functions[name] = self._bind(spec)
            except AttributeError:
                pass

    def _bind(self, spec: FunctionSpec):
        fn = getattr(self._native, spec.name)
        hints = get_type_hints(spec.func)
        sig = inspect.signature(spec.func)
        fn.argtypes = [_resolve_type(hints.get(p), self._tmap) for p in sig.parameters]
        fn.restype = _resolve_type(hints.get("return"), self._tmap)
        return fn

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        self._ensure_loaded()
        if name in self._functions:
            return self._functions[name]
        if name in _FUNCTION_REGISTRY:
            self._functions[name] = self._bind(_FUNCTION_REGISTRY[name])
            return self._functions[name]
        raise AttributeError(f"Function '{name}' not registered. Import the binding module first.")

    def __repr__(self):
        return f"<Library '{self._variant}' {'loaded' if self.is_loaded else 'not loaded'}>"


_LIBS: Dict[str, Library] = {}


def get_library(variant: str) -> Library:
    if variant not in _LIBS:
        _LIBS[variant] = Library(variant)
    return _LIBS[variant]


lib = get_library(DEFAULT_VARIANT)
