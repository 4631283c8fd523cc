"""Generate golden fixtures by running the reference's own Python code.

Run in a container where the reference checkout is readable:

    python tests/golden/make_golden.py /path/to/reference [--native-calls-only]

(or set QGPUSIM_REFERENCE to the checkout and omit the path).

It imports ``qgpusim/transpiler/passes.py`` and ``qgpusim/backends/custom/backend.py``
from the reference with small ``sys.modules`` stubs: Qiskit's base-pass and DAG
classes (the LQR algorithm only reads ``qubits``, ``topological_op_nodes()``,
``copy_empty_like()``, ``apply_operation_back()`` and node ``op/qargs/cargs``) and
CuPy (numpy stands in for it).  The native extension does not build (the shipped
``bindings.cpp`` has a syntax error), so ``backend.py`` takes its fallback executor.
That executor's ``permute_statevector`` gathers (``psi[idx_new]``) while the native
kernel scatters (``out[j] = in[i]``, qgpusim_cuda/src/kernels.cu:165-185); the two
differ for any non-involutive reorder.  The fixtures record the native (scatter)
semantics: ``permute_statevector`` is replaced by the scatter form before running.
The fallback's 2-qubit function also ignores the order of (q0, q1) (see
``native_order_2q``); it is called through the native index convention.

Outputs (all small, committed):
  schedules.json    -- LQR tile plans (qubits, layout, gate indices) per circuit
  states.npz        -- final statevectors of the reference executor (physical layout
                       of the last tile) for small circuits, complex128
  fusion.npz/.json  -- ``fuse_tile_ops`` results on seeded random op lists
  native_calls.json/.npz -- every call the reference's native branch of run_custom_backend
                       (backend.py:405-522) makes on its native extension for the state
                       cases, in each tile mode and precision (tests/golden/ref_harness.py)
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from frontierlabproject_b200 import circuits as C  # noqa: E402
from frontierlabproject_b200.circuit import QuantumCircuit, circuit_to_dag  # noqa: E402
from tests.golden.ref_harness import install_stubs, record_native_calls, save_trace  # noqa: E402


def scatter_permute(psi, layout_old, layout_new):
    """Native permute semantics: out[j] = in[i], j = sum_p bit_p(i) << map[p]."""
    n = len(layout_old)
    new_pos = {q: p for p, q in enumerate(layout_new)}
    mp = [new_pos[layout_old[p]] for p in range(n)]
    i = np.arange(1 << n, dtype=np.uint64)
    j = np.zeros_like(i)
    for p in range(n):
        j |= ((i >> np.uint64(p)) & np.uint64(1)) << np.uint64(mp[p])
    out = np.empty_like(psi)
    out[j] = psi
    return out


def native_order_2q(ref_fallback_2q):
    """The fallback's 2q function (backend.py:281-333) sorts the qubits and treats matrix
    index bit 0 as the lower qubit, so a gate with q0 > q1 gets its qubit roles swapped.
    The native kernel maps index b_q0 + 2*b_q1 (kernels.cu:108-114).  Calling the
    fallback with the bit-swapped matrix and sorted qubits gives the native semantics with
    the fallback's own arithmetic."""
    P = np.array([0, 2, 1, 3])

    def apply(psi, U, q0, q1, num_qubits):
        if q0 > q1:
            U = np.asarray(U)[np.ix_(P, P)]
            q0, q1 = q1, q0
        return ref_fallback_2q(psi, U, q0, q1, num_qubits)

    return apply


def schedule_record(qc, plan):
    # map node -> position in the input circuit by identity of (op, qargs)
    pos = {}
    for k, ins in enumerate(qc.data):
        pos[(id(ins.operation), tuple(ins.qubits))] = k
    tiles = []
    for t in plan:
        tiles.append({
            "tile_idx": t.tile_idx,
            "logical_qubits": list(t.logical_qubits),
            "layout": list(t.layout),
            "gates": [pos[(id(g.op), tuple(g.qargs))] for g in t.gates],
        })
    return tiles


def u_layers(n, depth, seed):
    """The reference benchmark circuit after Qiskit's default transpile merged RZ.RX into
    one ``u`` per qubit per layer (results/result.csv:6 shows 320 + 304 gates at n=20
    d=16), with the ``save_statevector`` directive the runner appends (runner.py:39-40)."""
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


NATIVE_CALL_CASES = ["random_layered_n10_d6_s1_nL6", "reference_random_n10_d4_s42_nL6", "reference_ghz_n9_nL4",
                     "reference_qft_n8_nL5", "qft_swaps_n9_nL5", "hea_n8_L3_nL5",
                     "random_layered_n8_d4_s5_save_nL6"]


def native_call_fixtures(ref_root, sched_cases):
    traces = record_native_calls(ref_root, {k: sched_cases[k] for k in NATIVE_CALL_CASES})
    save_trace(traces, os.path.join(HERE, "native_calls.json"), os.path.join(HERE, "native_calls.npz"))
    print(f"native calls: {len(traces)} traces")


def main(ref_root, native_calls_only=False):
    install_stubs()
    sys.path.insert(0, ref_root)
    import importlib
    passes = importlib.import_module("qgpusim.transpiler.passes")
    backend = importlib.import_module("qgpusim.backends.custom.backend")
    assert backend.USE_NATIVE is False
    backend.permute_statevector = scatter_permute
    backend.apply_2q_gate_cupy_fallback = native_order_2q(backend.apply_2q_gate_cupy_fallback)

    def ref_plan(qc, nL):
        lqr = passes.LazyQubitReordering(nL)
        lqr.run(circuit_to_dag(qc))
        return lqr.property_set["flat_tiling_plan"]

    # ---- schedules -------------------------------------------------------------------
    sched_cases = {
        "random_layered_n10_d6_s1_nL6": (C.random_layered(10, 6, 1), 6),
        "random_layered_n12_d8_s2_nL8": (C.random_layered(12, 8, 2), 8),
        "random_layered_n11_d5_s3_nL5": (C.random_layered(11, 5, 3), 5),
        "reference_random_n10_d4_s42_nL6": (C.reference_random(10, 4, 42), 6),
        "reference_ghz_n9_nL4": (C.reference_ghz(9), 4),
        "reference_qft_n8_nL5": (C.reference_qft(8), 5),
        "ghz_chain_n10_nL4": (C.ghz_chain(10), 4),
        "qft_swaps_n9_nL5": (C.qft(9, True), 5),
        "hea_n8_L3_nL5": (C.hea_ansatz(8, 3, np.linspace(-3, 3, 48)), 5),
        "random_layered_n20_d20_s0_nL14": (C.random_layered(20, 20, 0), 14),
        "ghz_chain_n32_nL16": (C.ghz_chain(32), 16),
        "ghz_chain_n32_nL20": (C.ghz_chain(32), 20),
        "ghz_chain_n32_nL24": (C.ghz_chain(32), 24),
        "qft_swaps_n30_nL16": (C.qft(30, True), 16),
        "qft_swaps_n30_nL20": (C.qft(30, True), 20),
        "qft_swaps_n30_nL24": (C.qft(30, True), 24),
        "random_layered_n30_d100_s0_nL20": (C.random_layered(30, 100, 0), 20),
        "random_layered_n33_d100_s0_nL20": (C.random_layered(33, 100, 0), 20),
        "u_layers_n20_d16_s42_nL16_save": (u_layers(20, 16, 42), 16),
        "u_layers_n25_d16_s42_nL16_save": (u_layers(25, 16, 42), 16),
    }
    save_case = C.random_layered(8, 4, 5)
    save_case.save_statevector()
    save_case.cx(0, 7)
    sched_cases["random_layered_n8_d4_s5_save_nL6"] = (save_case, 6)

    if native_calls_only:
        native_call_fixtures(ref_root, sched_cases)
        return
    schedules = {}
    for name, (qc, nL) in sched_cases.items():
        plan = ref_plan(qc, nL)
        schedules[name] = {"nL": nL, "num_qubits": qc.num_qubits, "num_ops": len(qc.data),
                           "tiles": schedule_record(qc, plan)}
        print(f"{name}: {len(plan)} tiles")
    with open(os.path.join(HERE, "schedules.json"), "w") as f:
        json.dump(schedules, f, separators=(",", ":"))

    # ---- statevectors from the reference executor --------------------------------------
    state_cases = ["random_layered_n10_d6_s1_nL6", "random_layered_n12_d8_s2_nL8",
                   "random_layered_n11_d5_s3_nL5", "reference_random_n10_d4_s42_nL6",
                   "reference_ghz_n9_nL4", "reference_qft_n8_nL5", "ghz_chain_n10_nL4",
                   "qft_swaps_n9_nL5", "hea_n8_L3_nL5", "random_layered_n8_d4_s5_save_nL6"]
    states = {}
    for name in state_cases:
        qc, nL = sched_cases[name]
        plan = ref_plan(qc, nL)
        backend.clear_gate_cache()
        psi = backend.run_custom_backend(qc, plan, "statevector", use_float32=False)
        states[name] = np.asarray(psi, dtype=np.complex128)
    np.savez_compressed(os.path.join(HERE, "states.npz"), **states)

    # ---- fuse_tile_ops ------------------------------------------------------------------
    rng = np.random.default_rng(7)
    fusion_inputs, fusion_meta = {}, []
    for case in range(12):
        nq = int(rng.integers(2, 6))
        nops = int(rng.integers(1, 25))
        ops = []
        for k in range(nops):
            if nq >= 2 and rng.random() < 0.4:
                q0, q1 = rng.choice(nq, size=2, replace=False)
                if rng.random() < 0.3 and ops and ops[-1][0] == "2q":
                    q0, q1 = ops[-1][1], ops[-1][2]
                U = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
                ops.append(("2q", int(q0), int(q1), U))
            else:
                q = int(rng.integers(0, nq))
                U = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
                ops.append(("1q", q, U))
        fused = backend.fuse_tile_ops(list(ops))
        meta = {"in": [], "out": []}
        for k, op in enumerate(ops):
            fusion_inputs[f"c{case}_in{k}"] = op[-1]
            meta["in"].append(list(op[:-1]))
        for k, op in enumerate(fused):
            fusion_inputs[f"c{case}_out{k}"] = np.asarray(op[-1])
            meta["out"].append(list(op[:-1]))
        fusion_meta.append(meta)
    np.savez_compressed(os.path.join(HERE, "fusion.npz"), **fusion_inputs)
    with open(os.path.join(HERE, "fusion.json"), "w") as f:
        json.dump(fusion_meta, f)
    native_call_fixtures(ref_root, sched_cases)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("QGPUSIM_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py /path/to/reference [--native-calls-only] (or set QGPUSIM_REFERENCE)")
    main(root, native_calls_only="--native-calls-only" in sys.argv)
