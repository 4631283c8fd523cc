"""Named circuits shared by the tests and the golden fixtures (same constructors as
tests/golden/make_golden.py)."""
import numpy as np

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.circuit import QuantumCircuit


def u_layers(n, depth, seed):
    import random
    rng = random.Random(seed)
    qc = QuantumCircuit(n)
    for _ in range(depth):
        for i in range(n):
            qc.u(2 * np.pi * rng.random(), 2 * np.pi * rng.random(), 2 * np.pi * rng.random(), i)
        for i in range(0, n - 1, 2):
            qc.cx(i, i + 1)
        for i in range(1, n - 1, 2):
            qc.cx(i, i + 1)
    qc.save_statevector()
    return qc


def _save_case():
    qc = C.random_layered(8, 4, 5)
    qc.save_statevector()
    qc.cx(0, 7)
    return qc


BUILDERS = {
    "random_layered_n10_d6_s1_nL6": lambda: C.random_layered(10, 6, 1),
    "random_layered_n12_d8_s2_nL8": lambda: C.random_layered(12, 8, 2),
    "random_layered_n11_d5_s3_nL5": lambda: C.random_layered(11, 5, 3),
    "reference_random_n10_d4_s42_nL6": lambda: C.reference_random(10, 4, 42),
    "reference_ghz_n9_nL4": lambda: C.reference_ghz(9),
    "reference_qft_n8_nL5": lambda: C.reference_qft(8),
    "ghz_chain_n10_nL4": lambda: C.ghz_chain(10),
    "qft_swaps_n9_nL5": lambda: C.qft(9, True),
    "hea_n8_L3_nL5": lambda: C.hea_ansatz(8, 3, np.linspace(-3, 3, 48)),
    "random_layered_n20_d20_s0_nL14": lambda: C.random_layered(20, 20, 0),
    "ghz_chain_n32_nL16": lambda: C.ghz_chain(32),
    "ghz_chain_n32_nL20": lambda: C.ghz_chain(32),
    "ghz_chain_n32_nL24": lambda: C.ghz_chain(32),
    "qft_swaps_n30_nL16": lambda: C.qft(30, True),
    "qft_swaps_n30_nL20": lambda: C.qft(30, True),
    "qft_swaps_n30_nL24": lambda: C.qft(30, True),
    "random_layered_n30_d100_s0_nL20": lambda: C.random_layered(30, 100, 0),
    "random_layered_n33_d100_s0_nL20": lambda: C.random_layered(33, 100, 0),
    "u_layers_n20_d16_s42_nL16_save": lambda: u_layers(20, 16, 42),
    "u_layers_n25_d16_s42_nL16_save": lambda: u_layers(25, 16, 42),
    "random_layered_n8_d4_s5_save_nL6": _save_case,
}

STATE_CASES = ["random_layered_n10_d6_s1_nL6", "random_layered_n12_d8_s2_nL8",
               "random_layered_n11_d5_s3_nL5", "reference_random_n10_d4_s42_nL6",
               "reference_ghz_n9_nL4", "reference_qft_n8_nL5", "ghz_chain_n10_nL4",
               "qft_swaps_n9_nL5", "hea_n8_L3_nL5", "random_layered_n8_d4_s5_save_nL6"]


def nl_of(name: str) -> int:
    return int(name.split("_nL")[1].split("_")[0])


def ops_of(qc):
    """Circuit -> ('1q', q, U) / ('2q', q0, q1, U) at logical qubits (unitary ops only)."""
    out = []
    for ins in qc.data:
        op = ins.operation
        if not hasattr(op, "to_matrix"):
            continue
        qs = [qc.find_bit(q).index for q in ins.qubits]
        U = op.to_matrix()
        out.append(("1q", qs[0], U) if len(qs) == 1 else ("2q", qs[0], qs[1], U))
    return out


# angles at which a rotation's cosine or sine (nearly) vanishes, and phases near 0 and 2 pi
ADVERSARIAL_ANGLES = (np.pi - 1e-7, np.pi + 1e-7, 1e-7, 2 * np.pi - 1e-7, np.pi - 1e-5, np.pi + 1e-4,
                      np.pi - 1e-3, 3 * np.pi - 1e-5)
ADVERSARIAL_PHASES = (1e-7, 2 * np.pi - 1e-7, np.pi + 1e-7, -1e-7, 1e-5)


def adversarial_angles(n, depth, seed):
    """Layers of RX / RY / RZ at angles where cos(t/2) or sin(t/2) is tiny, H on a few qubits,
    a CX ladder (no two rotations on one qubit fuse), and CP at phases near 0 and 2 pi: long
    runs of such gates land in one pass of the executor."""
    import random
    rng = random.Random(seed)
    from frontierlabproject_b200.circuit import QuantumCircuit
    qc = QuantumCircuit(n)
    for q in range(n):
        qc.h(q)
    for layer in range(depth):
        for q in range(n):
            t = rng.choice(ADVERSARIAL_ANGLES)
            g = rng.randrange(4)
            if g == 0:
                qc.rx(t, q)
            elif g == 1:
                qc.ry(t, q)
            elif g == 2:
                qc.rz(t, q)
            else:
                qc.rx(t, q)
                qc.ry(rng.choice(ADVERSARIAL_ANGLES), q)
        start = layer % 2
        for q in range(start, n - 1, 2):
            qc.cx(q, q + 1)
        for _ in range(max(1, n // 4)):
            a, b = rng.sample(range(n), 2)
            qc.cp(rng.choice(ADVERSARIAL_PHASES), a, b)
        qc.rx(np.pi - 1e-5, layer % n)
    return qc
