"""ruqu_b200 -- B200-native state-vector engine for ruqu-core's QAOA / VQE path.

The compute path is libruqu_cuda.so (hand-written sm_100a CUDA behind the C
ABI of include/ruqu_cuda.h).  This package is the host-side mirror of the
reference's API: ``QuantumState`` (crates/ruqu-core/src/state.rs),
``QuantumCircuit`` (circuit.rs), ``Gate`` (gate.rs), ``Simulator``
(simulator.rs), the types of types.rs and the QAOA / VQE drivers of
crates/ruqu-algorithms.

The public names load lazily: ``import ruqu_b200`` and the pure-host modules
(``ruqu_b200.workloads``, ``ruqu_b200.rng``, ``ruqu_b200.gate``) do not map
the CUDA library, so a CPU-only caller (the CPU baseline, workload
generators) never loads it.  The first access to a compute name
(``QuantumState``, ``Plan``, ``RQ_F32``, ...) loads libruqu_cuda.so and raises
ImportError if it is not built: there is no CPU fallback.
"""
from __future__ import annotations

import importlib

# public name -> submodule that defines it
_NAMES = {
    "RQ_EXEC_AUTO": "_capi", "RQ_EXEC_PER_GATE": "_capi", "RQ_EXEC_SWEEP": "_capi", "RQ_EXEC_SWEEP_TC": "_capi",
    "RQ_EXEC_SWEEP_TC_FAST": "_capi", "RQ_EXEC_SWEEP_TC16": "_capi", "RQ_F32": "_capi", "RQ_F64": "_capi",
    "QuantumCircuit": "circuit",
    "CircuitError": "error", "CudaError": "error", "DeviceTimeout": "error", "InvalidArgument": "error",
    "InvalidQubitIndex": "error", "InvalidStateVector": "error", "MemoryAllocationFailed": "error",
    "QuantumError": "error", "QubitLimitExceeded": "error",
    "Gate": "gate", "GateKind": "gate",
    "ShotResult": "simulator", "SimConfig": "simulator", "SimulationResult": "simulator", "Simulator": "simulator",
    "MAX_QUBITS": "state", "MAX_QUBITS_F32": "state", "Plan": "state", "QuantumState": "state",
    "set_device": "state",
    "Hamiltonian": "types", "MeasurementOutcome": "types", "NoiseModel": "types", "PauliOp": "types",
    "PauliString": "types", "SimulationMetrics": "types",
}

__all__ = sorted(_NAMES)


def __getattr__(name: str):
    mod = _NAMES.get(name)
    if mod is None:
        try:   # a submodule accessed as an attribute (ruqu_b200.workloads after `import ruqu_b200`)
            return importlib.import_module(f"{__name__}.{name}")
        except ModuleNotFoundError as e:
            if e.name != f"{__name__}.{name}":
                raise
            raise AttributeError(f"module {__name__!r} has no attribute {name!r}") from None
    value = getattr(importlib.import_module(f"{__name__}.{mod}"), name)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_NAMES))
