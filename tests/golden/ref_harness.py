"""Runs the reference's own executor code in this process (test infrastructure).

``install_stubs`` provides the small ``sys.modules`` stand-ins the reference's Python needs
here: Qiskit's base-pass / DAG names (the LQR pass only reads ``qubits``,
``topological_op_nodes()``, ``copy_empty_like()``, ``apply_operation_back()`` and node
``op/qargs/cargs``) and CuPy (numpy stands in for it).

``import_native_branch`` imports ``qgpusim/backends/custom/backend.py`` with a given module
installed as its native extension ``qgpusim.backends.custom.native.qgpusim_cuda``
(``backend.py:225-233``), so ``USE_NATIVE`` is True and ``run_custom_backend`` takes the
native branch (``backend.py:405-522``) -- the code path a drop-in replacement of the
extension serves.  ``recording_module`` is such a module: it records every call the branch
makes (constructor, ``permute``, ``apply_tile_*`` with their op lists, ``synchronize``,
``to_numpy``) and computes nothing.

The reference checkout is located by ``reference_root``; the tests that need it skip when it
is absent.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from frontierlabproject_b200.circuit import QuantumCircuit, circuit_to_dag  # noqa: E402


def reference_root(explicit: str = None):
    """The reference checkout to import (an explicit path, else $QGPUSIM_REFERENCE, else a
    directory named ``reference`` beside this repository), or None when it is absent."""
    for root in (explicit, os.environ.get("QGPUSIM_REFERENCE"), os.path.join(os.path.dirname(REPO), "reference")):
        if root and os.path.isfile(os.path.join(root, "qgpusim", "backends", "custom", "backend.py")):
            return root
    return None


def install_stubs():
    qiskit = types.ModuleType("qiskit")
    qiskit.QuantumCircuit = QuantumCircuit
    transpiler = types.ModuleType("qiskit.transpiler")
    basepasses = types.ModuleType("qiskit.transpiler.basepasses")

    class TransformationPass:
        def __init__(self):
            self.property_set = {}

    basepasses.TransformationPass = TransformationPass
    basepasses.AnalysisPass = TransformationPass
    dagmod = types.ModuleType("qiskit.dagcircuit")
    dagmod.DAGCircuit = object
    dagmod.DAGOpNode = object
    for name, mod in [("qiskit", qiskit), ("qiskit.transpiler", transpiler),
                      ("qiskit.transpiler.basepasses", basepasses), ("qiskit.dagcircuit", dagmod)]:
        sys.modules[name] = mod

    cupy = types.ModuleType("cupy")
    for attr in ("complex64", "complex128", "uint64", "int64", "asarray", "matmul", "zeros", "arange",
                 "ndarray"):
        setattr(cupy, attr, getattr(np, attr))
    cupy.asnumpy = np.asarray

    class _Pool:
        def free_all_blocks(self):
            pass

    cupy.get_default_memory_pool = lambda: _Pool()
    sys.modules["cupy"] = cupy


def import_passes(ref_root: str):
    install_stubs()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    return importlib.import_module("qgpusim.transpiler.passes")


def reference_plan(passes, qc, nL):
    lqr = passes.LazyQubitReordering(nL)
    lqr.run(circuit_to_dag(qc))
    return lqr.property_set["flat_tiling_plan"]


def import_native_branch(ref_root: str, native_module):
    """The reference's backend module, freshly imported with ``native_module`` as its
    native extension (USE_NATIVE = True)."""
    install_stubs()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    importlib.import_module("qgpusim.backends.custom")
    pkg = types.ModuleType("qgpusim.backends.custom.native")
    pkg.__path__ = []
    pkg.qgpusim_cuda = native_module
    sys.modules["qgpusim.backends.custom.native"] = pkg
    sys.modules["qgpusim.backends.custom.native.qgpusim_cuda"] = native_module
    sys.modules.pop("qgpusim.backends.custom.backend", None)
    backend = importlib.import_module("qgpusim.backends.custom.backend")
    sys.modules.pop("qgpusim.backends.custom.backend", None)  # later imports start fresh
    if not backend.USE_NATIVE:
        raise RuntimeError("the reference backend did not take the native module")
    return backend


def recording_module(trace: list):
    """A stand-in for the native extension that appends each call to ``trace``."""
    mod = types.ModuleType("qgpusim_cuda")

    class _SV:
        _np = np.complex128

        def __init__(self, num_qubits):
            self._n = int(num_qubits)
            trace.append({"call": type(self).__name__, "num_qubits": self._n})

        @property
        def num_qubits(self):
            return self._n

        @property
        def dim(self):
            return 1 << self._n

        def permute(self, layout_old, layout_new):
            trace.append({"call": "permute", "layout_old": [int(x) for x in layout_old],
                          "layout_new": [int(x) for x in layout_new]})

        def _tile(self, name, ops):
            rec = []
            for op in ops:
                U = np.array(np.asarray(op[-1]), copy=True)
                rec.append({"kind": op[0], "qubits": [int(x) for x in op[1:-1]], "U": U})
            trace.append({"call": name, "ops": rec})

        def apply_tile_cooperative(self, ops):
            self._tile("apply_tile_cooperative", ops)

        def apply_tile_graphed(self, ops):
            self._tile("apply_tile_graphed", ops)

        def apply_tile_dev(self, ops):
            self._tile("apply_tile_dev", ops)

        def synchronize(self):
            trace.append({"call": "synchronize"})

        def to_numpy(self):
            trace.append({"call": "to_numpy"})
            return np.zeros(1 << self._n, dtype=self._np)

        def reset(self):
            trace.append({"call": "reset"})

    class Statevector(_SV):
        _np = np.complex128

    class StatevectorF32(_SV):
        _np = np.complex64

    def apply_1q_gate(psi, U, target_qubit, num_qubits):
        trace.append({"call": "apply_1q_gate", "qubits": [int(target_qubit)], "U": np.array(U)})

    def apply_2q_gate(psi, U, q0, q1, num_qubits):
        trace.append({"call": "apply_2q_gate", "qubits": [int(q0), int(q1)], "U": np.array(U)})

    mod.Statevector = Statevector
    mod.StatevectorF32 = StatevectorF32
    mod.apply_1q_gate = apply_1q_gate
    mod.apply_2q_gate = apply_2q_gate
    return mod


def record_native_calls(ref_root: str, circuits: dict, modes=("cooperative", "graphed", "sequential"),
                        precisions=(False, True)) -> list:
    """Trace of the reference's native branch for each (circuit, tile mode, precision):
    circuits = {name: (qc, nL)}; schedules from the reference's own LQR pass."""
    passes = import_passes(ref_root)
    out = []
    for name, (qc, nl) in circuits.items():
        plan = reference_plan(passes, qc, nl)
        for f32 in precisions:
            for mode in modes:
                trace: list = []
                backend = import_native_branch(ref_root, recording_module(trace))
                backend.clear_gate_cache()
                backend.run_custom_backend(qc, plan, "statevector", use_float32=f32, tile_mode=mode)
                out.append({"case": name, "mode": mode, "f32": bool(f32), "calls": trace})
    return out


def save_trace(traces: list, json_path: str, npz_path: str) -> None:
    """Trace structure as JSON, matrices (deduplicated) as npz entries m0, m1, ..."""
    import json
    mats, index = {}, {}
    doc = []
    for t in traces:
        calls = []
        for c in t["calls"]:
            c2 = {k: v for k, v in c.items() if k not in ("ops", "U")}
            if "ops" in c:
                ops = []
                for op in c["ops"]:
                    U = np.ascontiguousarray(op["U"])
                    key = (U.dtype.str, U.shape, U.tobytes())
                    if key not in index:
                        index[key] = f"m{len(index)}"
                        mats[index[key]] = U
                    ops.append([op["kind"], op["qubits"], index[key]])
                c2["ops"] = ops
            calls.append(c2)
        doc.append({"case": t["case"], "mode": t["mode"], "f32": t["f32"], "calls": calls})
    with open(json_path, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    np.savez_compressed(npz_path, **mats)


def load_trace(json_path: str, npz_path: str) -> list:
    import json
    with open(json_path) as f:
        doc = json.load(f)
    with np.load(npz_path) as z:
        mats = {k: z[k] for k in z.files}
    for t in doc:
        for c in t["calls"]:
            if "ops" in c:
                c["ops"] = [{"kind": k, "qubits": q, "U": mats[m]} for k, q, m in c["ops"]]
    return doc
