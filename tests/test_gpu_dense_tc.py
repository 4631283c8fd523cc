"""Dense 64x64 unitaries on the tensor cores (qs_apply_dense6) against numpy in FP64."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.qgpusim_cuda import Statevector, StatevectorF32
from oracle import statevector as O

pytestmark = pytest.mark.gpu


def _unitary(rng, d=64):
    q, r = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _state(rng, n):
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (v / np.linalg.norm(v)).astype(np.complex64)


def _apply_ref(psi, U, qubits):
    """FP64: U on the listed qubits (row index sum_j b_{q_j} 2^j)."""
    n = psi.size.bit_length() - 1
    t = psi.astype(np.complex128).reshape([2] * n)          # axis a <-> qubit n-1-a
    axes = [n - 1 - q for q in reversed(qubits)]            # most significant of the 6 first
    rest = [a for a in range(n) if a not in axes]
    m = np.transpose(t, axes + rest).reshape(64, -1)
    m = U @ m
    out = np.transpose(m.reshape([2] * n), np.argsort(axes + rest))
    return out.reshape(-1)


def _infidelity(a, b):
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    return 1.0 - abs(np.vdot(a, b)) ** 2


@pytest.mark.parametrize("n", [13, 14, 18])
def test_dense6_low_qubits(n):
    rng = np.random.default_rng(n)
    U = _unitary(rng)
    psi = _state(rng, n)
    sv = StatevectorF32(n)
    sv.from_numpy(psi)
    sv.apply_dense(U)
    out = sv.to_numpy()
    ref = _apply_ref(psi, U, list(range(6)))
    assert _infidelity(ref, out) < 1e-6
    assert np.max(np.abs(out - ref)) < 1e-4 * np.max(np.abs(ref)) + 1e-6


def test_dense6_any_positions_and_inverse():
    rng = np.random.default_rng(7)
    n = 16
    U = _unitary(rng)
    q = [3, 7, 9, 12, 14, 1]
    psi = _state(rng, n)
    sv = StatevectorF32(n)
    sv.from_numpy(psi)
    sv.apply_dense(U, q)
    out = sv.to_numpy()
    assert _infidelity(_apply_ref(psi, U, q), out) < 1e-6
    sv.apply_dense(U.conj().T, q)
    back = sv.to_numpy()
    assert _infidelity(psi, back) < 2e-6


def test_dense6_after_queued_gates():
    # queued tile ops run before the dense unitary (materialised first)
    from frontierlabproject_b200 import gates as G
    rng = np.random.default_rng(3)
    n = 14
    U = _unitary(rng)
    psi = _state(rng, n)
    sv = StatevectorF32(n)
    sv.from_numpy(psi)
    H = np.array([[1, 1], [1, -1]], np.complex64) / np.sqrt(2)
    sv.apply_tile_graphed([("1q", 2, H), ("1q", 9, H)])
    sv.apply_dense(U)
    ref = psi.astype(np.complex128).copy()
    from oracle import statevector as O
    O.apply_1q(ref, H.astype(np.complex128), 2)
    O.apply_1q(ref, H.astype(np.complex128), 9)
    ref = _apply_ref(ref, U, list(range(6)))
    assert _infidelity(ref, sv.to_numpy()) < 1e-6


def test_dense6_rejects_unsupported_states():
    U = np.eye(64)
    with pytest.raises(RuntimeError, match="at least 13 qubits"):
        StatevectorF32(12).apply_dense(U)
    with pytest.raises(RuntimeError, match="complex64 states only"):
        Statevector(14).apply_dense(U)
    with pytest.raises(RuntimeError, match="64x64"):
        StatevectorF32(14).apply_dense(np.eye(4))


def _haar(d, rng):
    q, r = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _apply_block_ref(psi, qs, U):
    n = psi.size.bit_length() - 1
    m = len(qs)
    v = psi.reshape((2,) * n)
    vm = np.moveaxis(v, [n - 1 - q for q in qs][::-1], list(range(m)))
    sh = vm.shape
    vm[...] = (U @ vm.reshape(1 << m, -1)).reshape(sh)


@pytest.mark.parametrize("qs", [[0, 1, 2, 3, 4, 5], [3, 9, 1, 14, 7, 12], [15, 14, 13, 12, 11, 10], [6, 8],
                                [2], [0, 13, 6, 10], [9, 4, 15, 2, 11]])
def test_dense_block_any_positions(qs):
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    n = 16
    rng = np.random.default_rng(len(qs) * 7 + qs[0])
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    U = _haar(1 << len(qs), rng)
    sv = StatevectorF32(n)
    sv.from_numpy(psi.astype(np.complex64))
    ref = psi.copy()
    for _ in range(2):  # two launches in a row
        sv.apply_dense_block(qs, U)
        _apply_block_ref(ref, qs, U)
    out = sv.to_numpy().astype(np.complex128)
    assert O.infidelity(ref, out) <= 1e-5
    assert np.max(np.abs(out - ref)) <= 2e-5


def test_dense_block_after_a_relabel():
    # positions are layout positions: after permute() the block lands on the relabelled bits
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    n = 14
    rng = np.random.default_rng(3)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    sv = StatevectorF32(n)
    sv.from_numpy(psi.astype(np.complex64))
    lay = list(rng.permutation(n))
    sv.permute(list(range(n)), lay)
    ref = O.permute_scatter(psi, list(range(n)), lay)
    U = _haar(32, rng)
    sv.apply_dense_block([1, 12, 5, 0, 9], U)
    _apply_block_ref(ref, [1, 12, 5, 0, 9], U)
    assert O.infidelity(ref, sv.to_numpy()) <= 1e-5


@pytest.mark.parametrize("k", [4, 5, 6])
def test_dense_fusion_executor_matches_oracle(k):
    from frontierlabproject_b200.backend import run_custom_backend
    from frontierlabproject_b200.transpiler import tile_circuit
    qc = C.random_layered(18, 12, k)
    _, plan = tile_circuit(qc, 14)
    psi, met = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", dense_fusion=k,
                                  logical_order=True)
    assert 0 < met["dense_blocks"] < met["num_gates"]
    assert O.infidelity(O.simulate(qc), psi) <= 1e-5
