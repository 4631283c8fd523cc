"""Pass-manager factory, same signature as qgpusim/transpiler/pm.py:11-19."""
from __future__ import annotations

from typing import Optional, Tuple

from ..circuit import QuantumCircuit, circuit_to_dag, dag_to_circuit
from .passes import LazyQubitReordering


class PassManager:
    """Runs DAG passes in order on a circuit and returns the rewritten circuit."""

    def __init__(self):
        self._passes = []

    def append(self, passes) -> None:
        if isinstance(passes, (list, tuple)):
            self._passes.extend(passes)
        else:
            self._passes.append(passes)

    def run(self, qc: QuantumCircuit) -> QuantumCircuit:
        dag = circuit_to_dag(qc)
        for p in self._passes:
            dag = p.run(dag)
        return dag_to_circuit(dag)


def make_custom_pm(num_local_qubits: int, native: Optional[bool] = None) -> Tuple[PassManager, LazyQubitReordering]:
    lqr_pass = LazyQubitReordering(num_local_qubits, native)
    pm = PassManager()
    pm.append(lqr_pass)
    return pm, lqr_pass


def tile_circuit(qc: QuantumCircuit, num_local_qubits: int, native: Optional[bool] = None):
    """Convenience: (tiled circuit, tile plan) for ``qc`` at ``nL = num_local_qubits``
    (``native``: the C++ tiler; None = when the library loads)."""
    pm, lqr = make_custom_pm(num_local_qubits, native)
    tqc = pm.run(qc)
    return tqc, lqr.property_set["flat_tiling_plan"]
