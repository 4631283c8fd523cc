"""Dense 64x64 unitaries on the tensor cores (qs_apply_dense6) against numpy in FP64."""
import numpy as np
import pytest

from frontierlabproject_b200.qgpusim_cuda import Statevector, StatevectorF32

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
