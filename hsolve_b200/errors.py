"""hsolve's exception hierarchy (python/hsolve/__init__.py:50-130 in hsolve): one class per
hs::Error::Code, mapped by the code's snake_case name."""
from __future__ import annotations


class HsolveError(Exception):
    """Root of the error classes this package raises; ``code`` holds the snake_case name of the C++
    error code (hs::Error::Code) the error stands for."""

    code = "unknown"

    def __init__(self, message: str = "", code: str | None = None):
        super().__init__(message)
        if code is not None:
            self.code = code


class InvalidInputError(HsolveError, ValueError):
    code = "invalid_input"


class HsolveIOError(HsolveError, OSError):
    code = "io"


class NotHermitianError(HsolveError, ValueError):
    code = "not_hermitian"


class UnsupportedError(HsolveError, NotImplementedError):
    code = "unsupported"


class FactorizationFailedError(HsolveError, RuntimeError):
    code = "factorization_failed"


class SingularError(HsolveError, ArithmeticError):
    code = "singular"


class OutOfMemoryBudgetError(HsolveError, MemoryError):
    code = "out_of_memory_budget"


class NotConvergedError(HsolveError, RuntimeError):
    code = "not_converged"


class InternalError(HsolveError, RuntimeError):
    code = "internal"


class HsolveWarning(UserWarning):
    """Warning for a solve that returned pairs short of the requested tolerance; the report then
    carries success = False."""


ERROR_CLASSES = (InvalidInputError, HsolveIOError, NotHermitianError, UnsupportedError, FactorizationFailedError,
                 SingularError, OutOfMemoryBudgetError, NotConvergedError, InternalError)
_BY_CODE = {cls.code: cls for cls in ERROR_CLASSES}


def from_code(code: str, message: str) -> HsolveError:
    return _BY_CODE.get(code, InternalError)(message)
