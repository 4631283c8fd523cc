"""Gate matrices from their textbook definitions, in Qiskit's little-endian convention.

The reference obtains every matrix from ``op.to_matrix()`` (qgpusim/backends/custom/backend.py:46),
i.e. from Qiskit.  Qiskit is not available here; these are the standard
definitions.  For 2-qubit gates the matrix index is ``b_q0 + 2*b_q1`` with ``q0``
the first argument (the control of CX/CY/CP/CRZ), matching
qgpusim/backends/custom/qgpusim_cuda/src/kernels.cu:108-114.
"""
from __future__ import annotations

import cmath
import math
from typing import Sequence

import numpy as np

_S2 = 1.0 / math.sqrt(2.0)


def _controlled(u: np.ndarray) -> np.ndarray:
    """Control on bit 0 of the matrix index (q0), target on bit 1 (q1)."""
    m = np.eye(4, dtype=np.complex128)
    # indices with b_q0 = 1: 1 (b_q1=0) and 3 (b_q1=1)
    m[1, 1], m[1, 3] = u[0, 0], u[0, 1]
    m[3, 1], m[3, 3] = u[1, 0], u[1, 1]
    return m


def gate_matrix(name: str, params: Sequence[float] = ()) -> np.ndarray:
    p = [float(x) for x in params]
    c = np.complex128
    if name == "id":
        return np.eye(2, dtype=c)
    if name == "h":
        return np.array([[_S2, _S2], [_S2, -_S2]], dtype=c)
    if name == "x":
        return np.array([[0, 1], [1, 0]], dtype=c)
    if name == "y":
        return np.array([[0, -1j], [1j, 0]], dtype=c)
    if name == "z":
        return np.array([[1, 0], [0, -1]], dtype=c)
    if name == "s":
        return np.array([[1, 0], [0, 1j]], dtype=c)
    if name == "sdg":
        return np.array([[1, 0], [0, -1j]], dtype=c)
    if name == "t":
        return np.array([[1, 0], [0, cmath.exp(1j * math.pi / 4)]], dtype=c)
    if name == "tdg":
        return np.array([[1, 0], [0, cmath.exp(-1j * math.pi / 4)]], dtype=c)
    if name == "sx":
        return 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]], dtype=c)
    if name == "rx":
        a, b = math.cos(p[0] / 2), math.sin(p[0] / 2)
        return np.array([[a, -1j * b], [-1j * b, a]], dtype=c)
    if name == "ry":
        a, b = math.cos(p[0] / 2), math.sin(p[0] / 2)
        return np.array([[a, -b], [b, a]], dtype=c)
    if name == "rz":
        return np.array([[cmath.exp(-0.5j * p[0]), 0], [0, cmath.exp(0.5j * p[0])]], dtype=c)
    if name == "p":
        return np.array([[1, 0], [0, cmath.exp(1j * p[0])]], dtype=c)
    if name == "u":
        th, ph, la = p
        a, b = math.cos(th / 2), math.sin(th / 2)
        return np.array([[a, -cmath.exp(1j * la) * b],
                         [cmath.exp(1j * ph) * b, cmath.exp(1j * (ph + la)) * a]], dtype=c)
    if name == "cx":
        return _controlled(gate_matrix("x"))
    if name == "cy":
        return _controlled(gate_matrix("y"))
    if name == "cz":
        return np.diag([1, 1, 1, -1]).astype(c)
    if name == "cp":
        return np.diag([1, 1, 1, cmath.exp(1j * p[0])]).astype(c)
    if name == "crz":
        return _controlled(gate_matrix("rz", p))
    if name == "swap":
        return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=c)
    if name == "rzz":
        e0, e1 = cmath.exp(-0.5j * p[0]), cmath.exp(0.5j * p[0])
        return np.diag([e0, e1, e1, e0]).astype(c)
    raise ValueError(f"unknown gate: {name}")


GATE_ARITY = {
    "id": 1, "h": 1, "x": 1, "y": 1, "z": 1, "s": 1, "sdg": 1, "t": 1, "tdg": 1, "sx": 1,
    "rx": 1, "ry": 1, "rz": 1, "p": 1, "u": 1,
    "cx": 2, "cy": 2, "cz": 2, "cp": 2, "crz": 2, "swap": 2, "rzz": 2,
}

# Pauli generator G of each one-parameter rotation R(theta) = exp(-i theta G / 2).
ROTATION_GENERATOR = {"rx": "x", "ry": "y", "rz": "z"}
