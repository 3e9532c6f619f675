"""Exception hierarchy of the neighbour path, mirroring mlxlearn's
(reference src/mlxlearn/exceptions.py:1-168).

Capability mismatches (the request is understood but not served) are
``CapabilityError`` subclasses and also ``ValueError``/``TypeError`` as in
scikit-learn; a failure inside the CUDA library is a
``BackendExecutionError`` and is never re-run on the CPU.
"""
from __future__ import annotations

__all__ = [
    "MLXLearnError", "CapabilityError", "UnsupportedParameterError", "UnsupportedInputError",
    "SparseInputError", "DeviceError", "BackendExecutionError",
]


class MLXLearnError(Exception):
    """Base class for every error raised on purpose."""


class CapabilityError(MLXLearnError):
    """The request is understood but the CUDA path does not implement it."""

    def __init__(self, message: str, *, reason: str = "capability") -> None:
        super().__init__(message)
        self.reason = reason


class UnsupportedParameterError(CapabilityError, ValueError):
    """A constructor parameter value the brute-force Euclidean path does not cover."""

    def __init__(self, message: str, *, parameter: str, value: object = None) -> None:
        super().__init__(message, reason=f"unsupported-parameter:{parameter}")
        self.parameter = parameter
        self.value = value


class UnsupportedInputError(CapabilityError, ValueError):
    """Input data the path cannot handle (e.g. float64 values outside float32)."""

    def __init__(self, message: str, *, reason: str = "unsupported-input") -> None:
        super().__init__(message, reason=reason)


class SparseInputError(CapabilityError, TypeError):
    """Sparse input given to the dense-only path (message contains "sparse")."""

    def __init__(self, message: str) -> None:
        super().__init__(message, reason="sparse-input")


class DeviceError(MLXLearnError, RuntimeError):
    """No usable sm_100 device."""


class BackendExecutionError(MLXLearnError, RuntimeError):
    """The CUDA library failed; the status code is kept in ``status``."""

    def __init__(self, message: str, *, original: BaseException | None = None,
                 status: int | None = None) -> None:
        super().__init__(message)
        self.original = original
        self.status = status
