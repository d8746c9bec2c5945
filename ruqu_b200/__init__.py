"""ruqu_b200 -- B200-native state-vector engine for ruqu-core's QAOA / VQE path.

The compute path is libruqu_cuda.so (hand-written sm_100a CUDA behind the C
ABI of include/ruqu_cuda.h).  This package is the host-side mirror of the
reference's API: ``QuantumState`` (crates/ruqu-core/src/state.rs),
``QuantumCircuit`` (circuit.rs), ``Gate`` (gate.rs), ``Simulator``
(simulator.rs), the types of types.rs and the QAOA / VQE drivers of
crates/ruqu-algorithms.  Importing it fails if the library is not built.
"""
from ._capi import (RQ_EXEC_AUTO, RQ_EXEC_PER_GATE, RQ_EXEC_SWEEP, RQ_EXEC_SWEEP_TC, RQ_EXEC_SWEEP_TC_FAST, RQ_F32,
                    RQ_F64)
from .circuit import QuantumCircuit
from .error import (CircuitError, CudaError, DeviceTimeout, InvalidArgument, InvalidQubitIndex, InvalidStateVector,
                    MemoryAllocationFailed, QuantumError, QubitLimitExceeded)
from .gate import Gate, GateKind
from .simulator import ShotResult, SimConfig, SimulationResult, Simulator
from .state import MAX_QUBITS, MAX_QUBITS_F32, Plan, QuantumState, set_device
from .types import Hamiltonian, MeasurementOutcome, NoiseModel, PauliOp, PauliString, SimulationMetrics

__all__ = [
    "QuantumState", "Plan", "set_device", "QuantumCircuit", "Gate", "GateKind", "Simulator", "SimConfig", "SimulationResult",
    "ShotResult", "PauliOp", "PauliString", "Hamiltonian", "MeasurementOutcome", "SimulationMetrics",
    "NoiseModel",
    "QuantumError", "QubitLimitExceeded", "InvalidQubitIndex", "MemoryAllocationFailed", "InvalidStateVector",
    "CircuitError", "CudaError", "DeviceTimeout", "InvalidArgument", "MAX_QUBITS", "MAX_QUBITS_F32",
    "RQ_F32", "RQ_F64", "RQ_EXEC_AUTO", "RQ_EXEC_PER_GATE", "RQ_EXEC_SWEEP", "RQ_EXEC_SWEEP_TC",
    "RQ_EXEC_SWEEP_TC_FAST",
]
