"""Native op preparation (qs_prepare_ops / qs_gate_matrix) against the Python path of the
reference's native branch (per-gate matrices, fuse_tile_ops, packing), without a GPU."""
import ctypes

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200 import gates as G
from frontierlabproject_b200.backend import fuse_tile_ops, prepare_tile_ops, tile_ops_for
from frontierlabproject_b200.transpiler import tile_circuit
from tests.test_planner_cpu import _mixed


def test_gate_matrices_equal_the_python_table(native_lib):
    rng = np.random.default_rng(0)
    for name, gid in N.GATE_IDS.items():
        k = 3 if name == "u" else (1 if name in ("rx", "ry", "rz", "p", "cp", "crz", "rzz") else 0)
        for p in [np.zeros(3), np.full(3, np.pi), np.full(3, -np.pi)] + [rng.uniform(-7, 7, 3) for _ in range(50)]:
            ref = G.gate_matrix(name, p[:k])
            out = np.zeros(32)
            ar = ctypes.c_int()
            N.call("qs_gate_matrix", gid, p.ctypes.data, out.ctypes.data, ctypes.byref(ar))
            assert ar.value == G.GATE_ARITY[name]
            got = out[:2 * ref.size].view(np.complex128).reshape(ref.shape)
            np.testing.assert_array_equal(got, ref)  # entry for entry


def _fusing_circuit(n, seed):
    # runs of gates on one qubit / one ordered pair (fused), custom unitaries, all named gates
    from frontierlabproject_b200.circuit import QuantumCircuit
    rng = np.random.default_rng(seed)
    qc = QuantumCircuit(n)
    U2 = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
    for layer in range(4):
        for q in range(n):
            qc.h(q); qc.rz(float(rng.uniform(-3, 3)), q); qc.sx(q); qc.u(*rng.uniform(-3, 3, 3), q)
            qc.t(q); qc.sdg(q); qc.y(q); qc.p(float(rng.uniform(-3, 3)), q)
        for q in range(0, n - 1, 2):
            qc.cx(q, q + 1); qc.cx(q, q + 1); qc.cp(0.3, q, q + 1); qc.crz(0.7, q + 1, q)
            qc.unitary(U2, [q, q + 1]); qc.rzz(0.2, q, q + 1); qc.swap(q, q + 1); qc.cy(q + 1, q); qc.cz(q, q + 1)
    return qc


@pytest.mark.parametrize("code", [0, 1])
@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("case", ["random", "mixed", "fusing"])
def test_prepared_ops_equal_the_python_path(native_lib, code, fuse, case):
    qc = {"random": lambda: C.random_layered(14, 12, 3), "mixed": lambda: _mixed(12, 5),
          "fusing": lambda: _fusing_circuit(8, 2)}[case]()
    _, plan = tile_circuit(qc, 9)
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    dt = np.complex64 if code == 0 else np.complex128
    tol = 2e-6 if code == 0 else 1e-14  # products of fused matrices: last-bit differences
    total_in = total_out = 0
    for t in plan:
        batch, n_in = prepare_tile_ops(t, qmap, code, fuse)
        ops = tile_ops_for(t, qmap, dt)
        if fuse:
            ops = fuse_tile_ops(ops)
        assert n_in == len(tile_ops_for(t, qmap, dt))
        assert len(batch) == len(ops)
        total_in += n_in
        total_out += len(ops)
        for rec, op in zip(batch.arr, ops):
            assert rec["kind"] == (1 if op[0] == "1q" else 2)
            assert rec["q0"] == op[1] and (rec["q1"] == (op[2] if op[0] == "2q" else -1))
            d = 2 if op[0] == "1q" else 4
            got = np.ctypeslib.as_array(ctypes.cast(int(rec["U"]), ctypes.POINTER(ctypes.c_double if code else
                                                                                     ctypes.c_float)), (2 * d * d,))
            got = got.view(dt).reshape(d, d)
            np.testing.assert_allclose(got, np.asarray(op[-1], dtype=dt), rtol=0, atol=tol)
    if fuse and case == "fusing":
        assert total_out < total_in


def test_prepare_rejects_bad_input(native_lib):
    out = np.zeros(1, dtype=N.OP_DTYPE)
    mats = np.zeros(16, dtype=np.complex64)
    nout = ctypes.c_int()
    ids = np.array([99], dtype=np.int32)
    z = np.zeros(3)
    a = np.array([0], dtype=np.int32)
    b = np.array([-1], dtype=np.int32)
    rc = N.lib().qs_prepare_ops(0, 1, ids.ctypes.data, z.ctypes.data, a.ctypes.data, b.ctypes.data, None, 1,
                                out.ctypes.data, mats.ctypes.data, ctypes.byref(nout))
    assert rc == N.QS_ERR_INVALID and b"unknown gate id" in N.lib().qs_last_error()
    ids = np.array([N.GATE_IDS["cx"]], dtype=np.int32)
    rc = N.lib().qs_prepare_ops(0, 1, ids.ctypes.data, z.ctypes.data, a.ctypes.data, b.ctypes.data, None, 1,
                                out.ctypes.data, mats.ctypes.data, ctypes.byref(nout))
    assert rc == N.QS_ERR_INVALID and b"arity" in N.lib().qs_last_error()


@pytest.mark.parametrize("k", [2, 4, 5, 6])
def test_dense_block_plan_reproduces_the_tile(k):
    # the blocks' products, applied in order, equal the tile's gates applied one by one
    from frontierlabproject_b200.backend import plan_dense_blocks
    from oracle import statevector as O
    for qc, nl in ((_mixed(10, 4), 10), (C.random_layered(9, 6, 1), 9), (_fusing_circuit(8, 3), 8)):
        _, plan = tile_circuit(qc, nl)
        qmap = {q: qc.find_bit(q).index for q in qc.qubits}
        rng = np.random.default_rng(5)
        for t in plan:
            ops = tile_ops_for(t, qmap, np.complex128)
            n = qc.num_qubits
            psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
            want = psi.copy()
            for op in ops:
                if op[0] == "1q":
                    O.apply_1q(want, op[2], op[1])
                else:
                    O.apply_2q(want, op[3], op[1], op[2])
            blocks = plan_dense_blocks(ops, k)
            assert all(len(qs) <= k for qs, _ in blocks)
            got = psi.copy()
            for qs, U in blocks:
                # apply the block as a dense unitary on qubits qs (index sum_j b_qs[j] 2^j)
                m = len(qs)
                v = got.reshape((2,) * n)
                axes = [n - 1 - q for q in qs][::-1]  # block index bit m-1 .. 0
                vm = np.moveaxis(v, axes, list(range(m)))
                sh = vm.shape
                vm[...] = (U @ vm.reshape(1 << m, -1)).reshape(sh)
            np.testing.assert_allclose(got, want, atol=1e-12)
            if k >= 2:
                assert len(blocks) <= len(ops)
