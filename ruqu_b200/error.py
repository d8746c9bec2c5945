"""Error types (crates/ruqu-core/src/error.rs:8-26).

``QuantumError`` is the base class; its subclasses mirror the variants of
the reference enum, plus the device-side failures the GPU path adds.
"""
from __future__ import annotations


class QuantumError(Exception):
    code = -1


class QubitLimitExceeded(QuantumError):
    code = 1


class InvalidQubitIndex(QuantumError):
    code = 2


class MemoryAllocationFailed(QuantumError):
    code = 3


class InvalidStateVector(QuantumError):
    code = 4


class CircuitError(QuantumError):
    code = 5


class CudaError(QuantumError):
    code = 6


class DeviceTimeout(QuantumError):
    code = 7


class InvalidArgument(QuantumError):
    code = 8


_BY_CODE = {c.code: c for c in (QubitLimitExceeded, InvalidQubitIndex, MemoryAllocationFailed, InvalidStateVector,
                                CircuitError, CudaError, DeviceTimeout, InvalidArgument)}


def check(rc: int) -> None:
    """Raise the QuantumError subclass for a non-zero rq_status."""
    if rc != 0:
        from ._capi import last_error
        raise _BY_CODE.get(rc, QuantumError)(last_error())
