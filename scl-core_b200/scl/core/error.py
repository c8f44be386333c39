"""Error codes and exceptions (mirrors python/scl/core/error.py of scl-core).

Each library variant keeps its own thread-local error state, so
``check_error`` reads the message from the library that returned the code.
"""
from __future__ import annotations

SCL_OK = 0
SCL_ERROR_UNKNOWN = 1
SCL_ERROR_INTERNAL = 2
SCL_ERROR_OUT_OF_MEMORY = 3
SCL_ERROR_NULL_POINTER = 4
SCL_ERROR_INVALID_ARGUMENT = 10
SCL_ERROR_DIMENSION_MISMATCH = 11
SCL_ERROR_DOMAIN_ERROR = 12
SCL_ERROR_RANGE_ERROR = 13
SCL_ERROR_INDEX_OUT_OF_BOUNDS = 14
SCL_ERROR_TYPE_ERROR = 20
SCL_ERROR_TYPE_MISMATCH = 21
SCL_ERROR_NOT_IMPLEMENTED = 40
SCL_ERROR_FEATURE_UNAVAILABLE = 41
SCL_ERROR_NUMERICAL_ERROR = 50
SCL_ERROR_CONVERGENCE_ERROR = 54

_ERROR_MESSAGES = {
    SCL_ERROR_UNKNOWN: "Unknown error",
    SCL_ERROR_INTERNAL: "Internal error",
    SCL_ERROR_OUT_OF_MEMORY: "Out of memory",
    SCL_ERROR_NULL_POINTER: "Null pointer",
    SCL_ERROR_INVALID_ARGUMENT: "Invalid argument",
    SCL_ERROR_DIMENSION_MISMATCH: "Dimension mismatch",
    SCL_ERROR_INDEX_OUT_OF_BOUNDS: "Index out of bounds",
    SCL_ERROR_TYPE_MISMATCH: "Type mismatch",
    SCL_ERROR_NOT_IMPLEMENTED: "Not implemented",
    SCL_ERROR_FEATURE_UNAVAILABLE: "Feature unavailable",
    SCL_ERROR_CONVERGENCE_ERROR: "Convergence error",
}


class SCLError(Exception):
    """Base exception for all SCL errors (codes aligned with scl_core.h)."""

    def __init__(self, code: int, message: str | None = None):
        self.code = code
        if message is None:
            message = _ERROR_MESSAGES.get(code, f"Unknown error (code={code})")
        self.message = message
        super().__init__(f"SCL Error {code}: {message}")


class FeatureUnavailableError(SCLError):
    pass


def get_last_error(lib) -> tuple[int, str]:
    code = int(lib.scl_get_last_error_code())
    msg = lib.scl_get_last_error()
    return code, msg.decode() if isinstance(msg, bytes) else str(msg)


def check_error(code: int, context: str = "", lib=None) -> None:
    """Raise SCLError (with the library's thread-local message) unless code == SCL_OK."""
    if code == SCL_OK:
        return
    c_msg = _ERROR_MESSAGES.get(code, "error")
    if lib is not None:
        _, c_msg = get_last_error(lib)
    msg = f"{context}: {c_msg}" if context else c_msg
    cls = FeatureUnavailableError if code == SCL_ERROR_FEATURE_UNAVAILABLE else SCLError
    raise cls(code, msg)
