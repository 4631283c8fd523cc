"""Batched variational workload on the host: the batch program (planning, work items,
dependencies, gradient slots) emulated in FP64 against the oracle's adjoint gradients."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.batch import BatchShape, emulate, hea_batch
from oracle import statevector as O


def _oracle(inst):
    pc = inst.circuit
    L = sum(1 for g in pc.gates if g.name == "ry") // pc.num_qubits
    return O.adjoint_gradient(C.hea_ansatz(pc.num_qubits, L, inst.theta), inst.a, inst.b)


@pytest.mark.parametrize("shape", [BatchShape(m=9, small_max=6, chunk=2), BatchShape(m=10, small_max=0, chunk=3),
                                   BatchShape(m=13, small_max=13, chunk=4)])
def test_emulated_batch_matches_oracle(shape, native_lib):
    insts = hea_batch(7, n_range=(3, 12), l_range=(1, 3), seed=5)
    E, G = emulate(insts, shape)
    for inst, e, g in zip(insts, E, G):
        E_ref, g_ref = _oracle(inst)
        # float32 gate matrices, FP64 states and sums
        assert abs(e - E_ref) <= 1e-5 * max(1.0, abs(E_ref))
        np.testing.assert_allclose(g, g_ref, atol=2e-5)


def test_general_gates_and_fixed_controls(native_lib):
    # CX/CRZ with controls that stay unstaged, dense 2q gates, RX rotations (X generator)
    from frontierlabproject_b200.adjoint import ParamCircuit, ParamGate
    from frontierlabproject_b200.batch import Instance
    rng = np.random.default_rng(3)
    n = 12
    pc = ParamCircuit(n)
    k = 0
    for layer in range(3):
        for q in range(n):
            pc.gates.append(ParamGate(["rx", "ry", "rz"][(q + layer) % 3], (q,), k)); k += 1
        for q in range(0, n - 1, 2):
            pc.gates.append(ParamGate("cx", (n - 1 - q, q)))
        pc.gates.append(ParamGate("crz", (n - 1, 2), fixed=(0.7,)))
        pc.gates.append(ParamGate("swap", (1, 5)))
    pc.num_params = k
    inst = Instance(pc, rng.uniform(-np.pi, np.pi, k), rng.standard_normal(n), rng.standard_normal(n))
    E, G = emulate([inst], BatchShape(m=9, small_max=4, chunk=2))
    qc = pc.to_circuit(inst.theta)
    # reference: FP64 adjoint over the same gate list
    psi = O.simulate(qc)
    assert abs(E[0] - O.energy(psi, inst.a, inst.b)) <= 1e-5
    eps = 1e-6
    for j in range(0, k, 7):
        tp, tm = inst.theta.copy(), inst.theta.copy()
        tp[j] += eps
        tm[j] -= eps
        fd = (O.energy(O.simulate(pc.to_circuit(tp)), inst.a, inst.b) -
              O.energy(O.simulate(pc.to_circuit(tm)), inst.a, inst.b)) / (2 * eps)
        assert abs(G[0][j] - fd) <= 1e-4


def test_batch_argument_errors(native_lib):
    insts = hea_batch(2, n_range=(4, 5), l_range=(1, 1), seed=0)
    with pytest.raises(RuntimeError, match="m must be in 9..13"):
        emulate(insts, BatchShape(m=8))
    with pytest.raises(RuntimeError, match="threads must be 256 or 512"):
        emulate(insts, BatchShape(threads=100))


def test_autotune_reads_the_persisted_cache_without_timing(tmp_path):
    # a cache entry for this batch's size signature is used as is: no candidate is built or timed
    import json
    from frontierlabproject_b200 import batch as B
    insts = B.hea_batch(5, n_range=(6, 9), l_range=(2, 3), seed=3)
    path = str(tmp_path / "tune.json")
    key = B._cache_key(B._signature(insts))
    with open(path, "w") as f:
        json.dump({key: {"m": 12, "small_max": 11, "chunk": 2, "threads": 512, "blocks_per_sm": 0}}, f)
    B._TUNED.clear()
    shape = B.autotune(insts, shapes=[B.BatchShape(m=99)], cache_path=path)  # m=99 would fail if built
    assert shape == B.BatchShape(m=12, small_max=11, chunk=2, threads=512)
    B._TUNED.clear()
    B._store_cache(path, "other", B.BatchShape())
    with open(path) as f:
        assert set(json.load(f)) == {key, "other"}
