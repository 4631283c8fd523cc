"""Minimal quantum-circuit and DAG model for the tile executor.

The executor's drop-in surface (``run_custom_backend``, the LQR pass) reads only a
small part of Qiskit's circuit API: ``qc.num_qubits``, ``qc.qubits``,
``qc.find_bit(q).index`` and, per operation node, ``node.op.name``,
``node.op.params``, ``node.op.to_matrix()``, ``node.qargs`` and ``node.cargs``
(qgpusim/backends/custom/backend.py:370-451, qgpusim/transpiler/passes.py:359-420).
Qiskit is not a dependency of this package, so this module provides exactly
that surface.  Any object exposing the same attributes (a real Qiskit circuit
included) is accepted by the executor.

Operations without a ``to_matrix`` attribute (``save_statevector``, ``barrier``)
are kept in the circuit so the tiler sees them, and are skipped by the executor,
as qgpusim/backends/custom/backend.py:434-435 does.
"""
from __future__ import annotations

import copy as _copy
from dataclasses import dataclass, field
from typing import Iterable, List, NamedTuple, Optional, Sequence

import numpy as np

from . import gates as _gates


class Qubit:
    """An opaque qubit handle; its position in ``QuantumCircuit.qubits`` is its index."""

    __slots__ = ("_index",)

    def __init__(self, index: int):
        self._index = index

    def __repr__(self) -> str:
        return f"Qubit({self._index})"


class BitLocations(NamedTuple):
    index: int
    registers: list


class Gate:
    """A unitary operation with a matrix in Qiskit's little-endian convention.

    For a k-qubit gate applied to ``qargs = (q0, q1, ...)`` the matrix row/column
    index is ``b_q0 + 2*b_q1 + ...`` (qgpusim/backends/custom/qgpusim_cuda/src/kernels.cu:54-55).
    """

    def __init__(self, name: str, num_qubits: int, params: Sequence[float] = (), matrix=None):
        self.name = name
        self.num_qubits = num_qubits
        self.params = [float(p) for p in params]
        self._matrix = None if matrix is None else np.asarray(matrix, dtype=np.complex128)

    def to_matrix(self) -> np.ndarray:
        if self._matrix is not None:
            return self._matrix.copy()
        return _gates.gate_matrix(self.name, self.params)

    def inverse(self) -> "Gate":
        return Gate(self.name + "_dg", self.num_qubits, (), self.to_matrix().conj().T)

    def __repr__(self) -> str:
        p = f"({', '.join(f'{x:.6g}' for x in self.params)})" if self.params else ""
        return f"{self.name}{p}"


class Instruction:
    """A non-unitary directive (no ``to_matrix``): skipped by the executor."""

    def __init__(self, name: str, num_qubits: int, params: Sequence = ()):
        self.name = name
        self.num_qubits = num_qubits
        self.params = list(params)

    def __repr__(self) -> str:
        return self.name


@dataclass
class CircuitInstruction:
    operation: object
    qubits: tuple
    clbits: tuple = ()


class QuantumCircuit:
    """An ordered list of operations on ``num_qubits`` qubits."""

    def __init__(self, num_qubits: int):
        if num_qubits < 0:
            raise ValueError("num_qubits must be non-negative")
        self.qubits: List[Qubit] = [Qubit(i) for i in range(num_qubits)]
        self._index = {q: i for i, q in enumerate(self.qubits)}
        self.data: List[CircuitInstruction] = []
        self.global_phase = 0.0

    # -- Qiskit-compatible accessors -------------------------------------------------
    @property
    def num_qubits(self) -> int:
        return len(self.qubits)

    def find_bit(self, q: Qubit) -> BitLocations:
        return BitLocations(self._index[q], [])

    def copy(self) -> "QuantumCircuit":
        qc = QuantumCircuit(self.num_qubits)
        for ins in self.data:
            qc.data.append(CircuitInstruction(ins.operation,
                                              tuple(qc.qubits[self._index[q]] for q in ins.qubits),
                                              ins.clbits))
        qc.global_phase = self.global_phase
        return qc

    def __len__(self) -> int:
        return len(self.data)

    def size(self) -> int:
        return len(self.data)

    def count_ops(self) -> dict:
        out: dict = {}
        for ins in self.data:
            out[ins.operation.name] = out.get(ins.operation.name, 0) + 1
        return out

    # -- building --------------------------------------------------------------------
    def append(self, op, qargs: Iterable[int]) -> "QuantumCircuit":
        qs = tuple(self.qubits[int(q)] for q in qargs)
        if len(set(qs)) != len(qs):
            raise ValueError(f"duplicate qubit arguments for {op.name}: {list(qargs)}")
        for q in qargs:
            if not 0 <= int(q) < self.num_qubits:
                raise IndexError(f"qubit {q} out of range for a {self.num_qubits}-qubit circuit")
        self.data.append(CircuitInstruction(op, qs, ()))
        return self

    def _g(self, name, qargs, params=()):
        return self.append(Gate(name, len(qargs), params), qargs)

    def h(self, q): return self._g("h", (q,))
    def x(self, q): return self._g("x", (q,))
    def y(self, q): return self._g("y", (q,))
    def z(self, q): return self._g("z", (q,))
    def s(self, q): return self._g("s", (q,))
    def sdg(self, q): return self._g("sdg", (q,))
    def t(self, q): return self._g("t", (q,))
    def tdg(self, q): return self._g("tdg", (q,))
    def sx(self, q): return self._g("sx", (q,))
    def rx(self, theta, q): return self._g("rx", (q,), (theta,))
    def ry(self, theta, q): return self._g("ry", (q,), (theta,))
    def rz(self, theta, q): return self._g("rz", (q,), (theta,))
    def p(self, lam, q): return self._g("p", (q,), (lam,))
    def u(self, theta, phi, lam, q): return self._g("u", (q,), (theta, phi, lam))
    def cx(self, c, t): return self._g("cx", (c, t))
    def cy(self, c, t): return self._g("cy", (c, t))
    def cz(self, a, b): return self._g("cz", (a, b))
    def cp(self, lam, c, t): return self._g("cp", (c, t), (lam,))
    def crz(self, theta, c, t): return self._g("crz", (c, t), (theta,))
    def swap(self, a, b): return self._g("swap", (a, b))
    def rzz(self, theta, a, b): return self._g("rzz", (a, b), (theta,))

    def unitary(self, matrix, qargs, label: str = "unitary"):
        m = np.asarray(matrix, dtype=np.complex128)
        k = len(qargs)
        if m.shape != (1 << k, 1 << k):
            raise ValueError(f"unitary on {k} qubits needs a {1 << k}x{1 << k} matrix")
        return self.append(Gate(label, k, (), m), qargs)

    def save_statevector(self):
        """Directive on all qubits, as Qiskit-Aer's ``save_statevector`` (qgpusim/runner.py:39-40)."""
        return self.append(Instruction("save_statevector", self.num_qubits), range(self.num_qubits))

    def barrier(self, *qargs):
        qa = qargs if qargs else tuple(range(self.num_qubits))
        return self.append(Instruction("barrier", len(qa)), qa)

    def __repr__(self) -> str:
        return f"QuantumCircuit(num_qubits={self.num_qubits}, ops={len(self.data)})"


# --------------------------------------------------------------------------------------
# DAG view.  The LQR pass reads ``dag.qubits`` and ``dag.topological_op_nodes()``
# (qgpusim/transpiler/passes.py:359-366) and rebuilds a DAG with
# ``copy_empty_like`` / ``apply_operation_back`` (passes.py:401-416).
# --------------------------------------------------------------------------------------
class DAGOpNode:
    __slots__ = ("op", "qargs", "cargs", "_id")

    def __init__(self, op, qargs, cargs=(), node_id: int = 0):
        self.op = op
        self.qargs = tuple(qargs)
        self.cargs = tuple(cargs)
        self._id = node_id

    @property
    def name(self) -> str:
        return self.op.name

    def __repr__(self) -> str:
        return f"DAGOpNode({self.op!r}, id={self._id})"


class DAGCircuit:
    """Operation nodes in circuit order; circuit order is a valid topological order."""

    def __init__(self):
        self.qubits: List[Qubit] = []
        self._nodes: List[DAGOpNode] = []
        self.global_phase = 0.0

    def topological_op_nodes(self) -> List[DAGOpNode]:
        return list(self._nodes)

    def op_nodes(self) -> List[DAGOpNode]:
        return list(self._nodes)

    def copy_empty_like(self) -> "DAGCircuit":
        d = DAGCircuit()
        d.qubits = list(self.qubits)
        d.global_phase = self.global_phase
        return d

    def apply_operation_back(self, op, qargs=(), cargs=()) -> DAGOpNode:
        node = DAGOpNode(op, qargs, cargs, len(self._nodes))
        self._nodes.append(node)
        return node

    def size(self) -> int:
        return len(self._nodes)


def circuit_to_dag(qc: QuantumCircuit) -> DAGCircuit:
    d = DAGCircuit()
    d.qubits = list(qc.qubits)
    d.global_phase = getattr(qc, "global_phase", 0.0)
    for ins in qc.data:
        d.apply_operation_back(ins.operation, ins.qubits, ins.clbits)
    return d


def dag_to_circuit(dag: DAGCircuit) -> QuantumCircuit:
    qc = QuantumCircuit(0)
    qc.qubits = list(dag.qubits)
    qc._index = {q: i for i, q in enumerate(qc.qubits)}
    qc.global_phase = dag.global_phase
    for node in dag.topological_op_nodes():
        qc.data.append(CircuitInstruction(node.op, node.qargs, node.cargs))
    return qc
