"""GPU parity: the CUDA executor against the reference executor's fixtures and the oracle.

Tolerances: complex128 -> infidelity <= 1e-12 and |diff| <= 1e-12 per amplitude;
complex64 -> infidelity <= 1e-5 (per-amplitude |diff| <= 1e-5).  Permutations are
bit-exact.
"""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import fuse_tile_ops, run_custom_backend
from frontierlabproject_b200.qgpusim_cuda import (Statevector, StatevectorF32, apply_1q_gate, apply_2q_gate,
                                                  permute_scatter)
from frontierlabproject_b200.transpiler import tile_circuit
from oracle import statevector as O
from tests.cases import BUILDERS, STATE_CASES, nl_of

pytestmark = pytest.mark.gpu

MODES = ["cooperative", "graphed", "sequential"]
TOL = {True: 1e-5, False: 1e-12}


def _check(ref, psi, f32):
    assert O.infidelity(ref, psi) <= TOL[f32]
    assert np.max(np.abs(np.asarray(psi, np.complex128) - ref)) <= (1e-5 if f32 else 1e-12)


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", STATE_CASES)
def test_matches_reference_executor(name, mode, f32, golden_states):
    qc = BUILDERS[name]()
    _, plan = tile_circuit(qc, nl_of(name))
    psi, met = run_custom_backend(qc, plan, "statevector", use_float32=f32, tile_mode=mode)
    _check(golden_states[name], psi, f32)
    assert met["num_tiles"] == len(plan)


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("mode", MODES)
def test_config0_random_n20(mode, f32):
    # n=20, depth 20, nL=14, seed 0 (complex128 is the reference precision of this case)
    qc = C.random_layered(20, 20, 0)
    _, plan = tile_circuit(qc, 14)
    ref, layout = O.run_tile_plan(qc, plan, np.complex128)
    psi, met = run_custom_backend(qc, plan, "statevector", use_float32=f32, tile_mode=mode)
    _check(ref, psi, f32)
    assert met["num_reorders"] == sum(1 for a, b in zip([list(range(20))] + [t.layout for t in plan], [t.layout for t in plan]) if a != b)
    # logical order on request
    psi_l, _ = run_custom_backend(qc, plan, "statevector", use_float32=f32, tile_mode=mode, logical_order=True)
    _check(O.simulate(qc), psi_l, f32)


@pytest.mark.parametrize("cls", [Statevector, StatevectorF32])
@pytest.mark.parametrize("n", [6, 12, 17, 21])
def test_permute_bit_exact(cls, n):
    rng = np.random.default_rng(n)
    dt = np.complex128 if cls is Statevector else np.complex64
    psi = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dt)
    sv = cls(n)
    sv.from_numpy(psi)
    ref = psi.copy()
    layout = list(range(n))
    for _ in range(5):
        new = [int(x) for x in rng.permutation(n)]
        sv.permute(layout, new)
        ref = O.permute_scatter(ref, layout, new)
        layout = new
        if rng.random() < 0.5:
            assert np.array_equal(sv.to_numpy(), ref)
    assert np.array_equal(sv.to_numpy(), ref)


@pytest.mark.parametrize("dt", [np.complex64, np.complex128])
def test_reference_scatter_kernel_raw(dt):
    import torch
    n = 16
    rng = np.random.default_rng(1)
    psi = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dt)
    mp = [int(x) for x in rng.permutation(n)]
    a = torch.from_numpy(psi).cuda()
    b = torch.empty_like(a)
    permute_scatter(a, b, mp)
    torch.cuda.synchronize()
    layout_new = [mp.index(p) for p in range(n)]
    assert np.array_equal(b.cpu().numpy(), O.permute_scatter(psi, list(range(n)), layout_new))


@pytest.mark.parametrize("cls", [Statevector, StatevectorF32])
def test_per_gate_api(cls):
    import torch
    n = 11
    f32 = cls is StatevectorF32
    dt = np.complex64 if f32 else np.complex128
    rng = np.random.default_rng(5)
    psi = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n))
    psi /= np.linalg.norm(psi)
    sv = cls(n)
    sv.from_numpy(psi.astype(dt))
    ref = psi.copy()
    U1 = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))[0]
    U2 = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
    sv.apply_1q(3, U1); O.apply_1q(ref, U1, 3)
    sv.apply_2q(7, 2, U2); O.apply_2q(ref, U2, 7, 2)
    sv.apply_1q_dev(0, torch.from_numpy(U1.astype(dt)).cuda()); O.apply_1q(ref, U1, 0)
    sv.apply_2q_dev(4, 9, torch.from_numpy(U2.astype(dt)).cuda()); O.apply_2q(ref, U2, 4, 9)
    sv.apply_diagonal_1q(10, 1j, np.exp(0.3j)); O.apply_diagonal_1q(ref, 1j, np.exp(0.3j), 10)
    # a tile after a permute: ops are in the new layout
    sv.permute(list(range(n)), list(range(n))[::-1])
    ref = O.permute_scatter(ref, list(range(n)), list(range(n))[::-1])
    sv.apply_tile_cooperative([("1q", 1, U1), ("2q", 5, 0, U2)])
    O.apply_1q(ref, U1, 1); O.apply_2q(ref, U2, 5, 0)
    _check(ref, sv.to_numpy(), f32)
    assert abs(sv.norm_squared() - 1.0) < (1e-5 if f32 else 1e-12)
    with pytest.raises(RuntimeError, match="Invalid target qubit"):
        sv.apply_1q(n, U1)
    with pytest.raises(RuntimeError, match="q0 and q1 must be different"):
        sv.apply_2q(1, 1, U2)
    with pytest.raises(RuntimeError, match="layout_new is not a permutation"):
        sv.permute(list(range(n)), [0] * n)
    with pytest.raises(RuntimeError, match="apply_tile_dev: invalid q0"):
        sv.apply_tile_graphed([("1q", n, U1)])


@pytest.mark.parametrize("dt", [np.complex64, np.complex128])
def test_module_gate_functions(dt):
    import torch
    n = 13
    rng = np.random.default_rng(2)
    psi = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dt)
    t = torch.from_numpy(psi.copy()).cuda()
    U1 = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))[0]
    U2 = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
    apply_1q_gate(t, U1, 6, n)
    apply_2q_gate(t, U2, 12, 1, n)
    torch.cuda.synchronize()
    ref = psi.astype(np.complex128)
    O.apply_1q(ref, U1, 6)
    O.apply_2q(ref, U2, 12, 1)
    assert np.max(np.abs(t.cpu().numpy() - ref)) <= (1e-5 if dt == np.complex64 else 1e-12)


def test_known_answers_on_device():
    import torch
    # GHZ chain n=26 and QFT n=22 (with swaps) from |0...0>, complex64, cooperative mode
    qc = C.ghz_chain(26)
    _, plan = tile_circuit(qc, 16)
    sv = StatevectorF32(26)
    run_custom_backend(qc, plan, use_float32=True, tile_mode="cooperative", logical_order=True, sv=sv,
                       out=np.empty(1 << 26, np.complex64))
    v = sv.torch_view()
    assert abs(v[0].item() - 2 ** -0.5) < 1e-6 and abs(v[-1].item() - 2 ** -0.5) < 1e-6
    assert float((v.abs() ** 2).sum().item()) == pytest.approx(1.0, abs=1e-5)
    assert int((v.abs() > 1e-6).sum().item()) == 2
    qc = C.qft(22, True)
    _, plan = tile_circuit(qc, 20)
    psi, _ = run_custom_backend(qc, plan, use_float32=True, tile_mode="graphed", logical_order=True)
    assert np.max(np.abs(psi - 2 ** -11)) < 1e-6


def test_round_trip_large_n28():
    # U then U^dagger returns |0...0> (size-independent property at a large size)
    from frontierlabproject_b200.backend import tile_ops_for
    from frontierlabproject_b200.circuit import CircuitInstruction, QuantumCircuit
    qc = C.random_layered(28, 12, 3)
    inv = QuantumCircuit(28)
    for ins in reversed(qc.data):
        qs = tuple(inv.qubits[qc.find_bit(q).index] for q in ins.qubits)
        inv.data.append(CircuitInstruction(ins.operation.inverse(), qs))
    sv = StatevectorF32(28)
    for circ in (qc, inv):
        _, plan = tile_circuit(circ, 20)
        qmap = {q: circ.find_bit(q).index for q in circ.qubits}
        layout = list(range(28))
        for t in plan:
            if t.layout != layout:
                sv.permute(layout, t.layout)
                layout = t.layout
            sv.apply_tile_cooperative(fuse_tile_ops(tile_ops_for(t, qmap, np.complex64)))
        sv.permute(layout, list(range(28)))
    v = sv.torch_view()
    assert abs(abs(v[0].item()) - 1.0) < 1e-4
    assert float((v.abs() ** 2).sum().item()) == pytest.approx(1.0, abs=1e-4)
    st = sv.stats()
    assert st["sweeps"] > 0


def test_inner_product_and_norm():
    rng = np.random.default_rng(9)
    n = 15
    a = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n))
    b = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n))
    sa, sb = Statevector(n), Statevector(n)
    sa.from_numpy(a)
    sb.from_numpy(b)
    assert np.isclose(sa.norm_squared(), np.vdot(a, a).real, rtol=1e-12)
    assert np.isclose(sa.inner(sb), np.vdot(a, b), rtol=1e-12)


def test_reset_and_stats():
    sv = StatevectorF32(12)
    sv.apply_tile_cooperative([("1q", 0, np.array([[0, 1], [1, 0]]))])
    sv.reset()
    psi = sv.to_numpy()
    assert psi[0] == 1 and np.count_nonzero(psi) == 1
    assert sv.num_qubits == 12 and sv.dim == 4096
