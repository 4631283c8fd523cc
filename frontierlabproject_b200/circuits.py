"""Seeded workload circuits.

* ``random_layered`` -- the benchmark random circuit: per layer one gate per qubit
  drawn uniformly from {H, X, SX, RX(t), RZ(t)} with t ~ U[0, 2 pi), then CX on a
  random perfect matching of the qubits (one qubit idle when n is odd).
* ``ghz_chain`` -- H on q0, then CX q_i -> q_{i+1}.
* ``qft`` -- H plus controlled-phase 2 pi / 2^k ladders, then the final swaps.
* ``hea_ansatz`` -- hardware-efficient ansatz: per layer RY(t), RZ(t) on every qubit
  followed by a CZ ring.
* ``reference_random`` / ``reference_ghz`` / ``reference_qft`` -- the circuit
  families of qgpusim/circuits/builders.py:17-39 (RZ+RX per qubit plus brick-wall
  CX; CX fan-out from q0; QFT without swaps), used to reproduce the reference's
  published tile counts.
"""
from __future__ import annotations

import math
import random
from typing import List, Sequence, Tuple

import numpy as np

from .circuit import QuantumCircuit

ONE_QUBIT_SET = ("h", "x", "sx", "rx", "rz")


def random_layered(n: int, depth: int, seed: int) -> QuantumCircuit:
    rng = random.Random(seed)
    qc = QuantumCircuit(n)
    for _ in range(depth):
        for q in range(n):
            g = ONE_QUBIT_SET[rng.randrange(len(ONE_QUBIT_SET))]
            if g in ("rx", "rz"):
                getattr(qc, g)(2.0 * math.pi * rng.random(), q)
            else:
                getattr(qc, g)(q)
        perm = list(range(n))
        rng.shuffle(perm)
        for i in range(0, n - 1, 2):
            qc.cx(perm[i], perm[i + 1])
    return qc


def ghz_chain(n: int) -> QuantumCircuit:
    qc = QuantumCircuit(n)
    if n == 0:
        return qc
    qc.h(0)
    for i in range(n - 1):
        qc.cx(i, i + 1)
    return qc


def qft(n: int, do_swaps: bool = True) -> QuantumCircuit:
    """Textbook QFT on n qubits (qubit n-1 is the most significant)."""
    qc = QuantumCircuit(n)
    for j in range(n - 1, -1, -1):
        qc.h(j)
        for k in range(j - 1, -1, -1):
            qc.cp(2.0 * math.pi / (1 << (j - k + 1)), k, j)
    if do_swaps:
        for i in range(n // 2):
            qc.swap(i, n - 1 - i)
    return qc


def hea_ansatz(n: int, layers: int, thetas: Sequence[float]) -> QuantumCircuit:
    """RY/RZ on every qubit then a CZ ring, per layer; thetas ordered (layer, RY|RZ, qubit)."""
    th = np.asarray(thetas, dtype=np.float64).reshape(-1)
    if th.size != 2 * n * layers:
        raise ValueError(f"hea_ansatz needs {2 * n * layers} parameters, got {th.size}")
    qc = QuantumCircuit(n)
    i = 0
    for _ in range(layers):
        for q in range(n):
            qc.ry(float(th[i]), q); i += 1
        for q in range(n):
            qc.rz(float(th[i]), q); i += 1
        if n == 2:
            qc.cz(0, 1)
        elif n > 2:
            for q in range(n):
                qc.cz(q, (q + 1) % n)
    return qc


def hea_observable(n: int, seed: int) -> Tuple[np.ndarray, np.ndarray]:
    """Coefficients (a, b) of H = sum_i a_i Z_i Z_{i+1} + b_i X_i (periodic), a, b ~ N(0, 1)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n), rng.standard_normal(n)


def reference_random(n: int, depth: int, seed: int) -> QuantumCircuit:
    rng = random.Random(seed)
    qc = QuantumCircuit(n)
    for _ in range(max(1, depth)):
        for i in range(n):
            qc.rz(2 * math.pi * rng.random(), i)
            qc.rx(2 * math.pi * rng.random(), i)
        for i in range(0, n - 1, 2):
            qc.cx(i, i + 1)
        for i in range(1, n - 1, 2):
            qc.cx(i, i + 1)
    return qc


def reference_ghz(n: int) -> QuantumCircuit:
    qc = QuantumCircuit(n)
    qc.h(0)
    for i in range(1, n):
        qc.cx(0, i)
    return qc


def reference_qft(n: int) -> QuantumCircuit:
    return qft(n, do_swaps=False)


def build_circuit(circuit: str, n_qubits: int, depth: int = 1, seed: int = 0) -> QuantumCircuit:
    """Named builder, same names as qgpusim/circuits/builders.py:10-43 plus the benchmark families."""
    if circuit == "ghz":
        return reference_ghz(n_qubits)
    if circuit == "random":
        return reference_random(n_qubits, depth, seed)
    if circuit == "qft":
        return reference_qft(n_qubits)
    if circuit == "random_layered":
        return random_layered(n_qubits, depth, seed)
    if circuit == "ghz_chain":
        return ghz_chain(n_qubits)
    if circuit == "qft_swaps":
        return qft(n_qubits, True)
    raise ValueError(f"Unknown circuit type: {circuit}")
