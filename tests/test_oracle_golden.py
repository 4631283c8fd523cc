"""The CPU oracle pinned against fixtures produced by the reference's own executor."""
import json
import os

import numpy as np
import pytest

from oracle import statevector as O
from tests.cases import BUILDERS, STATE_CASES
from tests.conftest import GOLDEN


class _Tile:
    def __init__(self, rec, nodes):
        self.tile_idx = rec["tile_idx"]
        self.logical_qubits = rec["logical_qubits"]
        self.layout = rec["layout"]
        self.global_to_local_map = {q: i for i, q in enumerate(rec["logical_qubits"])}
        self.gates = [nodes[i] for i in rec["gates"]]


class _Node:
    def __init__(self, ins):
        self.op = ins.operation
        self.qargs = ins.qubits
        self.cargs = ins.clbits


def golden_plan(qc, rec):
    nodes = [_Node(ins) for ins in qc.data]
    return [_Tile(t, nodes) for t in rec["tiles"]]


@pytest.mark.parametrize("name", STATE_CASES)
def test_oracle_tile_loop_matches_reference_executor(name, schedules, golden_states):
    qc = BUILDERS[name]()
    plan = golden_plan(qc, schedules[name])
    psi, layout = O.run_tile_plan(qc, plan, np.complex128, fuse=True)
    ref = golden_states[name]
    assert layout == schedules[name]["tiles"][-1]["layout"]
    # fusion only reorders floating-point operations
    assert np.allclose(psi, ref, atol=1e-12, rtol=0)
    assert O.infidelity(ref, psi) <= 1e-12


@pytest.mark.parametrize("name", STATE_CASES)
def test_oracle_unfused_is_bitwise_reference(name, schedules, golden_states):
    # without fusion the oracle performs the reference fallback's exact arithmetic
    qc = BUILDERS[name]()
    plan = golden_plan(qc, schedules[name])
    psi, _ = O.run_tile_plan(qc, plan, np.complex128, fuse=False)
    assert np.allclose(psi, golden_states[name], atol=1e-14, rtol=0)


@pytest.mark.parametrize("name", STATE_CASES)
def test_golden_states_equal_logical_simulation(name, schedules, golden_states):
    # the reference executor's output is the logical state in the last tile's layout
    qc = BUILDERS[name]()
    logical = O.simulate(qc)
    layout = schedules[name]["tiles"][-1]["layout"]
    assert O.infidelity(O.to_layout(logical, layout), golden_states[name]) <= 1e-12


def test_fusion_fixtures():
    meta = json.load(open(os.path.join(GOLDEN, "fusion.json")))
    z = np.load(os.path.join(GOLDEN, "fusion.npz"))
    for c, m in enumerate(meta):
        ops = [tuple(d) + (z[f"c{c}_in{k}"],) for k, d in enumerate(m["in"])]
        fused = O.fuse_ops(ops)
        assert [list(o[:-1]) for o in fused] == m["out"]
        for k, o in enumerate(fused):
            assert np.allclose(o[-1], z[f"c{c}_out{k}"], atol=1e-12)


def test_permute_map_messages():
    with pytest.raises(RuntimeError, match="layout_new is not a permutation"):
        O.permute_map([0, 1, 2], [0, 0, 2])
    with pytest.raises(RuntimeError, match="layout_old/layout_new must have length num_qubits"):
        O.permute_map([0, 1], [0, 1, 2])
    with pytest.raises(RuntimeError, match="layout_new contains invalid qubit id"):
        O.permute_map([0, 1, 2], [0, 1, 3])


def test_known_answers():
    from frontierlabproject_b200 import circuits as C
    n = 9
    ghz = O.simulate(C.ghz_chain(n))
    want = np.zeros(1 << n, complex)
    want[0] = want[-1] = 2 ** -0.5
    assert np.allclose(ghz, want, atol=1e-14)
    q = O.simulate(C.qft(n, True))
    assert np.allclose(q, np.full(1 << n, 2 ** (-n / 2)), atol=1e-13)
    # QFT of a basis state |x>: amplitudes exp(2 pi i x y / N) / sqrt(N)
    x = 0b101101011
    psi0 = np.zeros(1 << n, complex)
    psi0[x] = 1
    out = O.simulate(C.qft(n, True), psi0=psi0)
    y = np.arange(1 << n)
    assert np.allclose(out, np.exp(2j * np.pi * x * y / (1 << n)) / 2 ** (n / 2), atol=1e-12)


def test_adjoint_gradient_matches_finite_differences():
    from frontierlabproject_b200 import circuits as C
    n, L = 5, 2
    rng = np.random.default_rng(3)
    th = rng.uniform(-np.pi, np.pi, 2 * n * L)
    a, b = C.hea_observable(n, 4)
    E, g = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
    assert np.isclose(E, O.energy(O.simulate(C.hea_ansatz(n, L, th)), a, b))
    h = 1e-5
    fd = np.empty_like(th)
    for i in range(th.size):
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (O.energy(O.simulate(C.hea_ansatz(n, L, tp)), a, b) -
                 O.energy(O.simulate(C.hea_ansatz(n, L, tm)), a, b)) / (2 * h)
    assert np.allclose(g, fd, atol=1e-8)
