"""Known-answer tests of the reference, as data.

Each case restates one test of crates/ruqu-core/tests/test_state.rs or
test_simulator.rs (cited per case): the gate sequence it applies and the
values it asserts, at the reference's tolerance of 1e-10
(test_state.rs:5, test_simulator.rs:5).  The expected values are the
analytic ones those tests assert; they pin the oracle (tests/test_oracle_kats.py)
and, through the C ABI, the GPU engine (tests/test_gpu_parity.py).

Steps: ("g", kind, q0, q1, angle) applies a gate (kind = rq_gate_kind code),
("reset", q) calls reset_qubit.  Checks: ("amp", i, re, im),
("prob", i, p), ("probs_zero_except", [indices]), ("expect", ops, v),
("ham", [(coeff, ops)], v), ("prob_qubit", q, p), ("total", 1.0).
"""
import math

H, X, Y, Z, S, SDG, T, TDG, RX, RY, RZ, PHASE, CNOT, CZ, SWAP, RZZ = range(16)
PX, PY, PZ = 1, 2, 3
s2 = 0.7071067811865476
TS = "crates/ruqu-core/tests/test_state.rs"
TSIM = "crates/ruqu-core/tests/test_simulator.rs"


def g(kind, q0, q1=0, angle=0.0):
    return ("g", kind, q0, q1, angle)


CASES = [
    dict(name="initial_1q", ref=f"{TS}:16-23", n=1, steps=[], checks=[("prob", 0, 1.0), ("prob", 1, 0.0)]),
    dict(name="initial_2q", ref=f"{TS}:26-35", n=2, steps=[], checks=[("prob", 0, 1.0), ("probs_zero_except", [0])]),
    dict(name="initial_3q", ref=f"{TS}:38-46", n=3, steps=[], checks=[("prob", 0, 1.0), ("probs_zero_except", [0])]),
    dict(name="hadamard_superposition", ref=f"{TS}:70-77", n=1, steps=[g(H, 0)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.5)]),
    dict(name="hadamard_amplitudes", ref=f"{TS}:80-89", n=1, steps=[g(H, 0)],
         checks=[("amp", 0, s2, 0.0), ("amp", 1, s2, 0.0)]),
    dict(name="double_hadamard", ref=f"{TS}:92-100", n=1, steps=[g(H, 0), g(H, 0)],
         checks=[("prob", 0, 1.0), ("prob", 1, 0.0)]),
    dict(name="hadamard_on_qubit_1_of_2", ref=f"{TS}:103-113", n=2, steps=[g(H, 1)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.0), ("prob", 2, 0.5), ("prob", 3, 0.0)]),
    dict(name="x_flips", ref=f"{TS}:120-127", n=1, steps=[g(X, 0)], checks=[("prob", 0, 0.0), ("prob", 1, 1.0)]),
    dict(name="double_x", ref=f"{TS}:130-137", n=1, steps=[g(X, 0), g(X, 0)], checks=[("prob", 0, 1.0)]),
    dict(name="x_on_second_qubit", ref=f"{TS}:140-148", n=2, steps=[g(X, 1)], checks=[("prob", 0, 0.0), ("prob", 2, 1.0)]),
    dict(name="y_on_zero", ref=f"{TS}:155-165", n=1, steps=[g(Y, 0)],
         checks=[("prob", 0, 0.0), ("prob", 1, 1.0), ("amp", 1, 0.0, 1.0)]),
    dict(name="z_on_zero", ref=f"{TS}:172-178", n=1, steps=[g(Z, 0)], checks=[("prob", 0, 1.0)]),
    dict(name="z_phase", ref=f"{TS}:181-194", n=1, steps=[g(H, 0), g(Z, 0)],
         checks=[("amp", 0, s2, 0.0), ("amp", 1, -s2, 0.0)]),
    dict(name="z_on_one", ref=f"{TS}:197-207", n=1, steps=[g(X, 0), g(Z, 0)],
         checks=[("prob", 0, 0.0), ("prob", 1, 1.0), ("amp", 1, -1.0, 0.0)]),
    dict(name="bell", ref=f"{TS}:214-224", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.0), ("prob", 2, 0.0), ("prob", 3, 0.5)]),
    dict(name="bell_amplitudes", ref=f"{TS}:227-237", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("amp", 0, s2, 0.0), ("amp", 3, s2, 0.0)]),
    dict(name="bell_phi_minus", ref=f"{TS}:240-251", n=2, steps=[g(H, 0), g(CNOT, 0, 1), g(Z, 0)],
         checks=[("amp", 0, s2, None), ("amp", 3, -s2, None)]),
    dict(name="bell_psi_plus", ref=f"{TS}:254-268", n=2, steps=[g(H, 0), g(CNOT, 0, 1), g(X, 0)],
         checks=[("prob", 0, 0.0), ("prob", 1, 0.5), ("prob", 2, 0.5), ("prob", 3, 0.0)]),
    dict(name="ghz3", ref=f"{TS}:275-292", n=3, steps=[g(H, 0), g(CNOT, 0, 1), g(CNOT, 1, 2)],
         checks=[("prob", 0, 0.5), ("prob", 7, 0.5), ("probs_zero_except", [0, 7])]),
    dict(name="ghz4", ref=f"{TS}:295-307", n=4, steps=[g(H, 0), g(CNOT, 0, 1), g(CNOT, 1, 2), g(CNOT, 2, 3)],
         checks=[("prob", 0, 0.5), ("prob", 15, 0.5), ("probs_zero_except", [0, 15])]),
    dict(name="swap", ref=f"{TS}:314-325", n=2, steps=[g(X, 1), g(SWAP, 0, 1)],
         checks=[("prob", 0, 0.0), ("prob", 1, 1.0), ("prob", 2, 0.0), ("prob", 3, 0.0)]),
    dict(name="swap_both_same", ref=f"{TS}:328-334", n=2, steps=[g(SWAP, 0, 1)], checks=[("prob", 0, 1.0)]),
    dict(name="double_swap", ref=f"{TS}:337-345", n=2, steps=[g(X, 1), g(SWAP, 0, 1), g(SWAP, 0, 1)],
         checks=[("prob", 2, 1.0)]),
    dict(name="rx_zero_identity", ref=f"{TS}:352-357", n=1, steps=[g(RX, 0, 0, 0.0)], checks=[("prob", 0, 1.0)]),
    dict(name="rx_pi_is_x", ref=f"{TS}:360-368", n=1, steps=[g(RX, 0, 0, math.pi)],
         checks=[("prob", 0, 0.0), ("prob", 1, 1.0)]),
    dict(name="ry_pi_flips", ref=f"{TS}:371-378", n=1, steps=[g(RY, 0, 0, math.pi)], checks=[("prob", 1, 1.0)]),
    dict(name="rz_preserves_probability", ref=f"{TS}:381-386", n=1, steps=[g(RZ, 0, 0, 1.234)],
         checks=[("prob", 0, 1.0)]),
    dict(name="rx_half_pi", ref=f"{TS}:389-398", n=1, steps=[g(RX, 0, 0, math.pi / 2)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.5)]),
    dict(name="ry_half_pi", ref=f"{TS}:401-409", n=1, steps=[g(RY, 0, 0, math.pi / 2)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.5)]),
    dict(name="cz_on_11", ref=f"{TS}:416-426", n=2, steps=[g(X, 0), g(X, 1), g(CZ, 0, 1)],
         checks=[("amp", 3, -1.0, None), ("prob", 3, 1.0)]),
    dict(name="cz_on_01", ref=f"{TS}:429-436", n=2, steps=[g(X, 1), g(CZ, 0, 1)], checks=[("amp", 2, 1.0, None)]),
    dict(name="expect_z_zero", ref=f"{TS}:556-563", n=1, steps=[], checks=[("expect", [(0, PZ)], 1.0)]),
    dict(name="expect_z_one", ref=f"{TS}:566-574", n=1, steps=[g(X, 0)], checks=[("expect", [(0, PZ)], -1.0)]),
    dict(name="expect_z_plus", ref=f"{TS}:577-585", n=1, steps=[g(H, 0)], checks=[("expect", [(0, PZ)], 0.0)]),
    dict(name="expect_x_plus", ref=f"{TS}:588-596", n=1, steps=[g(H, 0)], checks=[("expect", [(0, PX)], 1.0)]),
    dict(name="expect_x_minus", ref=f"{TS}:599-608", n=1, steps=[g(X, 0), g(H, 0)], checks=[("expect", [(0, PX)], -1.0)]),
    dict(name="expect_zz_bell", ref=f"{TS}:611-620", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("expect", [(0, PZ), (1, PZ)], 1.0)]),
    dict(name="expect_xx_bell", ref=f"{TS}:623-632", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("expect", [(0, PX), (1, PX)], 1.0)]),
    dict(name="expect_yy_bell", ref=f"{TS}:635-644", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("expect", [(0, PY), (1, PY)], -1.0)]),
    dict(name="expect_identity", ref=f"{TS}:647-654", n=2, steps=[g(H, 0), g(RX, 1, 0, 1.5)],
         checks=[("expect", [], 1.0)]),
    dict(name="hamiltonian_simple", ref=f"{TS}:661-674", n=1, steps=[], checks=[("ham", [(1.0, [(0, PZ)])], 1.0)]),
    dict(name="hamiltonian_two_terms", ref=f"{TS}:677-699", n=2, steps=[],
         checks=[("ham", [(0.5, [(0, PZ)]), (0.5, [(1, PZ)])], 1.0)]),
    dict(name="hamiltonian_after_flip", ref=f"{TS}:702-725", n=2, steps=[g(X, 0)],
         checks=[("ham", [(1.0, [(0, PZ)]), (1.0, [(1, PZ)])], 0.0)]),
    dict(name="normalization_after_gates", ref=f"{TS}:732-742", n=3,
         steps=[g(H, 0), g(CNOT, 0, 1), g(RX, 2, 0, 1.23), g(RZ, 0, 0, 0.456), g(RY, 1, 0, 2.1), g(CZ, 0, 2)],
         checks=[("total", 1.0)]),
    dict(name="normalization_many_gates", ref=f"{TS}:745-757", n=4,
         steps=[g(H, 0), g(H, 1), g(H, 2), g(H, 3), g(CNOT, 0, 1), g(CNOT, 2, 3), g(SWAP, 1, 2), g(RX, 0, 0, 0.7),
                g(RY, 3, 0, 1.2)],
         checks=[("total", 1.0)]),
    dict(name="reset_qubit", ref=f"{TS}:764-770", n=1, steps=[g(X, 0), ("reset", 0)], checks=[("prob", 0, 1.0)]),
    dict(name="reset_from_superposition", ref=f"{TS}:773-779", n=1, steps=[g(H, 0), ("reset", 0)],
         checks=[("prob", 0, 1.0)]),
    dict(name="reset_one_of_entangled", ref=f"{TS}:782-791", n=2, steps=[g(H, 0), g(CNOT, 0, 1), ("reset", 0)],
         checks=[("prob_qubit", 0, 0.0)]),
    dict(name="s_on_plus", ref=f"{TS}:880-891", n=1, steps=[g(H, 0), g(S, 0)],
         checks=[("amp", 0, s2, 0.0), ("amp", 1, 0.0, s2)]),
    dict(name="t_phase", ref=f"{TS}:894-905", n=1, steps=[g(H, 0), g(T, 0)],
         checks=[("amp", 0, s2, None), ("amp", 1, s2 * math.cos(math.pi / 4), s2 * math.sin(math.pi / 4))]),
    dict(name="rzz_zero_identity", ref=f"{TS}:912-922", n=2, steps=[g(H, 0), g(H, 1), g(RZZ, 0, 1, 0.0)],
         checks=[("prob", 0, 0.25), ("prob", 1, 0.25), ("prob", 2, 0.25), ("prob", 3, 0.25)]),
    dict(name="superdense_00", ref=f"{TS}:976-987", n=2, steps=[g(H, 0), g(CNOT, 0, 1), g(CNOT, 0, 1), g(H, 0)],
         checks=[("prob", 0, 1.0)]),
    dict(name="superdense_01", ref=f"{TS}:990-1001", n=2,
         steps=[g(H, 0), g(CNOT, 0, 1), g(X, 0), g(CNOT, 0, 1), g(H, 0)], checks=[("prob", 2, 1.0)]),
    dict(name="superdense_10", ref=f"{TS}:1004-1015", n=2,
         steps=[g(H, 0), g(CNOT, 0, 1), g(Z, 0), g(CNOT, 0, 1), g(H, 0)], checks=[("prob", 1, 1.0)]),
    dict(name="superdense_11", ref=f"{TS}:1018-1029", n=2,
         steps=[g(H, 0), g(CNOT, 0, 1), g(X, 0), g(Z, 0), g(CNOT, 0, 1), g(H, 0)], checks=[("prob", 3, 1.0)]),
    dict(name="simulator_bell", ref=f"{TSIM}:154-163", n=2, steps=[g(H, 0), g(CNOT, 0, 1)],
         checks=[("prob", 0, 0.5), ("prob", 1, 0.0), ("prob", 2, 0.0), ("prob", 3, 0.5)]),
    dict(name="simulator_ghz", ref=f"{TSIM}:186-196", n=3, steps=[g(H, 0), g(CNOT, 0, 1), g(CNOT, 1, 2)],
         checks=[("prob", 0, 0.5), ("prob", 7, 0.5), ("probs_zero_except", [0, 7])]),
    dict(name="simulator_qft_like", ref=f"{TSIM}:412-427", n=3,
         steps=[g(H, 0), g(RZ, 0, 0, math.pi / 4), g(RZ, 0, 0, math.pi / 2), g(H, 1), g(RZ, 1, 0, math.pi / 4),
                g(H, 2), g(SWAP, 0, 2)],
         checks=[("total", 1.0)]),
    dict(name="simulator_many_gates", ref=f"{TSIM}:430-446", n=5,
         steps=[g(H, q) for q in range(5)] + [g(CNOT, i, i + 1) for i in range(4)] +
               [g(RZ, i, 0, 0.3 * i) for i in range(5)],
         checks=[("total", 1.0)]),
]

# State-vector fidelity KATs (test_state.rs:798-830): (gates_a, gates_b, n, expected)
FIDELITY = [
    dict(ref=f"{TS}:798-801", n=2, a=[], b=[], value=1.0),
    dict(ref=f"{TS}:804-809", n=1, a=[], b=[g(X, 0)], value=0.0),
    dict(ref=f"{TS}:812-818", n=1, a=[], b=[g(H, 0)], value=0.5),
]

EPS = 1e-10
