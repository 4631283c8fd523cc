"""Native gate fusion (qs_fuse_ops) against the reference's own fusion results (golden fixtures
recorded from qgpusim's fuse_tile_ops) and against the Python restatement on random op lists.
Host only."""
import ctypes
import json
import os

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200.backend import fuse_tile_ops
from frontierlabproject_b200.qgpusim_cuda import _OpBatch
from tests.conftest import REPO

GOLDEN = os.path.join(REPO, "tests", "golden")


def _unpack(batch, code):
    dt = np.complex64 if code == N.QS_C64 else np.complex128
    item = np.dtype(dt).itemsize
    out = []
    for rec in batch.arr:
        k = 4 if rec["kind"] == N.QS_OP_1Q else 16
        m = np.frombuffer((ctypes.c_char * (k * item)).from_address(int(rec["U"])), dtype=dt).copy()
        if rec["kind"] == N.QS_OP_1Q:
            out.append(("1q", int(rec["q0"]), m.reshape(2, 2)))
        else:
            out.append(("2q", int(rec["q0"]), int(rec["q1"]), m.reshape(4, 4)))
    return out


def _same(a, b, tol):
    assert [o[:-1] for o in a] == [o[:-1] for o in b]
    for x, y in zip(a, b):
        np.testing.assert_allclose(x[-1], y[-1], rtol=0, atol=tol)


@pytest.mark.parametrize("code", [N.QS_C64, N.QS_C128])
def test_native_fusion_matches_reference_fixtures(native_lib, code):
    dt = np.complex64 if code == N.QS_C64 else np.complex128
    meta = json.load(open(os.path.join(GOLDEN, "fusion.json")))
    z = np.load(os.path.join(GOLDEN, "fusion.npz"))
    for c, m in enumerate(meta):
        ops = [tuple(d) + (np.asarray(z[f"c{c}_in{k}"], dt),) for k, d in enumerate(m["in"])]
        fused = _unpack(_OpBatch(ops, code).fused(), code)
        assert [list(o[:-1]) for o in fused] == m["out"]
        for k, o in enumerate(fused):
            np.testing.assert_allclose(o[-1], z[f"c{c}_out{k}"], rtol=0, atol=1e-5 if code == N.QS_C64 else 1e-12)


def _random_ops(rng, n, count, dt):
    ops = []
    for _ in range(count):
        if rng.random() < 0.6:
            q = int(rng.integers(0, n))
            U = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))[0]
            ops.append(("1q", q, U.astype(dt)))
        else:
            q0, q1 = (int(x) for x in rng.choice(n, 2, replace=False))
            U = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
            ops.append(("2q", q0, q1, U.astype(dt)))
    return ops


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("code", [N.QS_C64, N.QS_C128])
def test_native_fusion_equals_python(native_lib, seed, code):
    dt = np.complex64 if code == N.QS_C64 else np.complex128
    rng = np.random.default_rng(seed)
    # few qubits: many fusable runs, interleaved 1q / 2q on shared qubits, reversed pairs
    ops = _random_ops(rng, 3 + seed % 3, 60, dt)
    ops += [("2q", 0, 1, ops[0][-1] if ops[0][0] == "2q" else np.eye(4, dtype=dt)), ("2q", 1, 0, np.eye(4, dtype=dt))]
    want = fuse_tile_ops(list(ops))
    got = _unpack(_OpBatch(ops, code).fused(), code)
    _same(got, want, 2e-5 if code == N.QS_C64 else 1e-12)


def test_native_fusion_edge_cases(native_lib):
    dt = np.complex64
    assert len(_OpBatch([], N.QS_C64).fused()) == 0
    H = (np.array([[1, 1], [1, -1]]) / np.sqrt(2)).astype(dt)
    got = _unpack(_OpBatch([("1q", 2, H), ("1q", 2, H)], N.QS_C64).fused(), N.QS_C64)
    assert len(got) == 1 and np.allclose(got[0][-1], np.eye(2), atol=1e-6)
    with pytest.raises(RuntimeError, match="q0 == q1"):
        _OpBatch([("2q", 1, 1, np.eye(4, dtype=dt))], N.QS_C64).fused()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["cooperative", "graphed"])
def test_run_custom_backend_native_fusion(mode):
    # the reference's circuit family fuses RZ.RX runs: native and Python fusion give one state
    from frontierlabproject_b200 import circuits as C
    from frontierlabproject_b200.backend import run_custom_backend
    from frontierlabproject_b200.transpiler import tile_circuit
    from oracle import statevector as O
    qc = C.reference_random(14, 6, 3)
    _, plan = tile_circuit(qc, 10)
    a, ma = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode=mode)
    b, mb = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode=mode, native_fusion=True)
    assert ma["fusion_ratio"] == mb["fusion_ratio"] > 1.0
    assert O.infidelity(a, b) <= 1e-6
    assert np.max(np.abs(a - b)) <= 1e-5
