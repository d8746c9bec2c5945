"""Host-side checks that need no GPU: the C-ABI library loads and exports every
symbol include/ruqu_cuda.h declares, the Python mirror of the reference API
(circuit builder, gates, types) behaves like the reference, and the seeded
workload generators are deterministic and valid."""
import ctypes
import math
import os
import re

import numpy as np

import oracle
import ruqu_b200 as rq
from ruqu_b200 import Gate, GateKind, QuantumCircuit, rng, workloads
from ruqu_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^RQ_API\s+[\w\s\*]+?\b(rq_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = _declared_symbols()
    assert len(names) >= 25
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers every declared entry point too
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)


def test_abi_header_compiles_as_c_and_cpp(tmp_path):
    """include/*.h is the drop-in boundary for C and C++ callers (and Rust / cgo binding
    generators): it must compile on its own as C99 and as C++11, warning-free."""
    import shutil
    import subprocess
    for cc, std, ext in (("gcc", "-std=c99", "c"), ("g++", "-std=c++11", "cpp")):
        exe = shutil.which(cc)
        if exe is None:
            continue
        for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
            if not h.endswith(".h"):
                continue
            src = tmp_path / f"use_{h}.{ext}"
            src.write_text(f'#include "{h}"\nint main(void) {{ return 0; }}\n')
            r = subprocess.run([exe, std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                                "-I" + os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
            assert r.returncode == 0, (cc, h, r.stderr)


def test_host_uniform_matches_oracle_and_numpy():
    for seed, stream in ((0, 0), (42, 0), (2**63 + 5, 3), (17, 1)):
        u = rng.uniforms(seed, stream, 0, 9)
        for i in range(9):
            assert u[i] == oracle.uniform(seed, stream, i) == _capi.lib.rq_uniform(seed, stream, i)


# ---- circuit builder (crates/ruqu-core/tests/test_simulator.rs:15-138) ----

def test_circuit_builder_counts():
    c = QuantumCircuit(3)
    assert c.num_qubits() == 3 and c.gate_count() == 0
    c.h(0).h(1).h(2).cnot(0, 1).cnot(1, 2)
    assert c.gate_count() == 5
    c1 = QuantumCircuit(1).h(0).x(0).y(0).z(0).s(0).t(0).rx(0, .5).ry(0, .5).rz(0, .5)
    assert c1.gate_count() == 9
    c2 = QuantumCircuit(2).cnot(0, 1).cz(0, 1).swap(0, 1).rzz(0, 1, .5)
    assert c2.gate_count() == 4
    c3 = QuantumCircuit(3).h(0).h(1).h(2).measure_all()
    assert c3.gate_count() >= 6
    assert QuantumCircuit(2).reset(0).barrier().gate_count() == 2


def test_circuit_depth():
    assert QuantumCircuit(1).h(0).depth() == 1
    assert QuantumCircuit(3).h(0).h(1).h(2).depth() == 1
    assert QuantumCircuit(1).h(0).x(0).z(0).depth() == 3
    assert QuantumCircuit(2).h(0).cnot(0, 1).h(1).depth() == 3
    # barrier levels all qubits (circuit.rs:161-167)
    assert QuantumCircuit(2).h(0).h(0).barrier().h(1).depth() == 3


def test_gate_matrices_and_qubits():
    s2 = 1 / math.sqrt(2)
    assert np.allclose(Gate.H(0).matrix_1q(), [[s2, s2], [s2, -s2]])
    assert np.allclose(Gate.Y(0).matrix_1q(), [[0, -1j], [1j, 0]])
    assert np.allclose(Gate.Rx(0, math.pi).matrix_1q(), [[0, -1j], [-1j, 0]], atol=1e-15)
    assert np.allclose(Gate.Rz(0, math.pi).matrix_1q(), [[-1j, 0], [0, 1j]], atol=1e-15)
    cnot = Gate.CNOT(0, 1).matrix_2q()
    assert cnot[2, 3] == 1 and cnot[3, 2] == 1 and cnot[0, 0] == 1
    assert Gate.H(3).qubits() == [3] and Gate.CNOT(1, 2).qubits() == [1, 2] and Gate.Barrier().qubits() == []
    assert Gate.Measure(0).is_non_unitary() and not Gate.H(0).is_non_unitary()
    assert Gate.CNOT(0, 1).matrix_1q() is None and Gate.H(0).matrix_2q() is None
    for k in (GateKind.H, GateKind.X, GateKind.Rx, GateKind.Ry, GateKind.Rz, GateKind.Phase):
        m = Gate(k, 0, angle=0.9).matrix_1q()
        assert np.allclose(m @ m.conj().T, np.eye(2), atol=1e-14)


def test_estimate_memory():
    assert rq.QuantumState.estimate_memory(1) == 32
    assert rq.QuantumState.estimate_memory(10) == 16384
    assert rq.QuantumState.estimate_memory(20) == 16_777_216
    assert rq.QuantumState.estimate_memory(3, "f32") == 64
    assert rq.QuantumState.estimate_memory(10, "f32") == 8192


# ---- workloads ----

def test_random_layer_circuit_shape():
    g = workloads.random_layer_circuit(20, 40, 0)
    n1 = sum(1 for x in g if x[0] in (GateKind.Rz, GateKind.Rx))
    n2 = sum(1 for x in g if x[0] == GateKind.CNOT)
    assert n1 == 1600 and n2 == 380          # 20 qubits x 40 layers; 10/9 CNOTs per layer
    g30 = workloads.random_layer_circuit(30, 20, 1)
    assert sum(1 for x in g30 if x[0] == GateKind.CNOT) == 290
    assert g == workloads.random_layer_circuit(20, 40, 0)
    assert all(0 <= x[3] < 2 * math.pi for x in g if x[0] != GateKind.CNOT)


def test_random_3regular_graphs():
    st = rng.Stream(123, 2)
    for n in range(12, 27, 2):
        e = workloads.random_3regular_graph(n, st)
        assert len(e) == 3 * n // 2
        deg = np.bincount(np.array(e).ravel(), minlength=n)
        assert (deg == 3).all()
        assert len(set(e)) == len(e) and all(i < j for i, j in e)


def test_qaoa_instances_deterministic():
    a = workloads.qaoa_instances(16, 7)
    b = workloads.qaoa_instances(16, 7)
    assert [x["n"] for x in a] == [x["n"] for x in b]
    assert all(12 <= x["n"] <= 24 and x["n"] % 2 == 0 for x in a)
    assert all((0 <= x["gammas"]).all() and (x["gammas"] < math.pi).all() for x in a)
    assert all((0 <= x["betas"]).all() and (x["betas"] < math.pi / 2).all() for x in a)


def test_pauli_hamiltonian():
    c, s = workloads.pauli_hamiltonian(16, 200, 3)
    assert len(c) == 200 and len(s) == 200
    ops = [o for t in s for _, o in t]
    assert set(ops) <= {1, 2, 3}
    assert 0.6 < len(ops) / (200 * 16) < 0.9      # 3/4 non-identity
    assert abs(np.mean(c)) < 0.3 and 0.7 < np.std(c) < 1.3


def test_rng_box_muller_moments():
    z = rng.Stream(9, 4).normal(20000)
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.03


def test_uniforms_keys_equal_the_per_key_stream():
    """rng.uniforms_keys (draw k of many keys at once, the shots of a distributed sample)
    equals draw k of each key's own stream."""
    import numpy as np
    from ruqu_b200.rng import uniforms, uniforms_keys
    keys = np.array([0, 1, 42, 2**63 + 5, 2**64 - 1], dtype=np.uint64)
    for k in (0, 1, 2, 7, 1000001):
        want = np.array([uniforms(int(s), 0, k, 1)[0] for s in keys])
        assert np.array_equal(uniforms_keys(keys, 0, k), want)
