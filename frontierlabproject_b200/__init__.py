"""B200-native tile executor for lazy-qubit-reordering statevector schedules.

Drop-in surface (names of the reference ``qgpusim`` package):
  transpiler: ``LazyQubitReordering``, ``Tile``, ``make_custom_pm``
  backend:    ``run_custom_backend``, ``fuse_tile_ops``
  native:     ``qgpusim_cuda.Statevector``, ``StatevectorF32``, ``apply_1q_gate``, ``apply_2q_gate``
The native parts need ``libqsim_b200.so`` (``python -m frontierlabproject_b200.build``).
"""
from .circuit import QuantumCircuit, circuit_to_dag, dag_to_circuit
from . import circuits, gates
from .transpiler import LazyQubitReordering, Tile, make_custom_pm, tile_circuit

__all__ = ["QuantumCircuit", "circuit_to_dag", "dag_to_circuit", "circuits", "gates",
           "LazyQubitReordering", "Tile", "make_custom_pm", "tile_circuit"]
