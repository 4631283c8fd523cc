"""Planner, encoder and ABI checks that need no GPU (host emulation of the device program)."""
import ctypes
import os
import re

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.qgpusim_cuda import _OpBatch
from oracle import statevector as O
from tests.cases import ops_of
from tests.conftest import REPO


def _emulate(qc, code, m=None, k=3):
    dt = np.complex64 if code == 0 else np.complex128
    n = qc.num_qubits
    b = _OpBatch(ops_of(qc), code)
    psi = np.zeros(1 << n, dtype=dt)
    psi[0] = 1
    cfg = N.QsConfig(m or (13 if code == 0 else 12), k, 4, 0)
    sw, ph = ctypes.c_int(), ctypes.c_int()
    N.call("qs_plan_info", n, code, b.ptr, len(b), ctypes.byref(cfg), ctypes.byref(sw), ctypes.byref(ph))
    N.call("qs_plan_emulate", n, code, b.ptr, len(b), ctypes.byref(cfg), psi.ctypes.data)
    return psi, sw.value, ph.value


def _mixed(n, seed):
    qc = C.random_layered(n, 6, seed)
    rng = np.random.default_rng(seed)
    qc.cz(0, n - 1); qc.cp(0.3, 2, n - 3); qc.swap(1, n - 2); qc.rzz(0.7, 0, 3); qc.crz(0.4, 4, 1)
    qc.cx(n - 1, 0); qc.y(2); qc.s(3); qc.t(n - 1); qc.ry(0.2, 5); qc.cy(2, min(6, n - 1))
    U = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
    qc.unitary(U, [3, 5]); qc.unitary(U, [n - 1, 2])
    return qc


@pytest.mark.parametrize("code", [0, 1])
@pytest.mark.parametrize("n", [6, 9, 13, 16])
def test_plan_emulation_matches_oracle(native_lib, code, n):
    qc = _mixed(n, n)
    psi, sweeps, phases = _emulate(qc, code)
    ref = O.simulate(qc)
    tol = 1e-6 if code == 0 else 1e-13
    assert O.infidelity(ref, psi) <= tol
    assert sweeps >= 1 and phases >= sweeps


@pytest.mark.parametrize("k", [1, 2, 3, 4])
@pytest.mark.parametrize("m", [7, 10, 13])
def test_plan_config_sweep(native_lib, m, k):
    qc = _mixed(15, 7)
    psi, _, _ = _emulate(qc, 0, m=m, k=k)
    assert O.infidelity(O.simulate(qc), psi) <= 1e-6


@pytest.mark.parametrize("n", [6, 8, 13, 17, 20])
def test_inplace_permutation_bit_exact(native_lib, n):
    rng = np.random.default_rng(n)
    for _ in range(4):
        perm = rng.permutation(n).astype(np.int32)
        psi = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
        # scatter with map_old_to_new = perm
        layout_new = [int(np.where(perm == p)[0][0]) for p in range(n)]
        ref = O.permute_scatter(psi.copy(), list(range(n)), layout_new)
        out = psi.copy()
        sw = ctypes.c_int()
        cfg = N.QsConfig(13, 3, 4, 0)
        N.call("qs_perm_emulate", n, 0, perm.ctypes.data, ctypes.byref(cfg), out.ctypes.data, ctypes.byref(sw))
        assert np.array_equal(out, ref)
        assert sw.value <= 4


def test_config2_sweep_count(native_lib):
    # the n=30 depth-100 benchmark circuit: far fewer sweeps than the reference schedule's
    # 67 tiles + 66 reorders + 1
    qc = C.random_layered(30, 100, 0)
    b = _OpBatch(ops_of(qc), 0)
    sw, ph = ctypes.c_int(), ctypes.c_int()
    N.call("qs_plan_info", 30, 0, b.ptr, len(b), None, ctypes.byref(sw), ctypes.byref(ph))
    assert sw.value < 100


def test_abi_exports_every_declared_symbol(native_lib):
    header = open(os.path.join(REPO, "include", "qsim_b200.h")).read()
    declared = set(re.findall(r"QS_API\s+[\w\s\*]*?\b(qs_\w+)\s*\(", header))
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(native_lib, name), name
    assert declared == set(N.exported_symbols())


def test_abi_validation_messages(native_lib):
    h = ctypes.c_void_p()
    assert native_lib.qs_create(10, 7, ctypes.byref(h)) != 0
    assert b"dtype" in native_lib.qs_last_error()
    assert native_lib.qs_create(0, 0, ctypes.byref(h)) != 0
    assert b"num_qubits" in native_lib.qs_last_error()
    with pytest.raises(RuntimeError, match="apply_tile_dev: q0 == q1"):
        b = _OpBatch([("2q", 1, 1, np.eye(4))], 0)
        N.call("qs_plan_info", 8, 0, b.ptr, 1, None, None, None)
    with pytest.raises(RuntimeError, match="apply_tile_dev: invalid q0"):
        b = _OpBatch([("1q", 9, np.eye(2))], 0)
        N.call("qs_plan_info", 8, 0, b.ptr, 1, None, None, None)
    with pytest.raises(RuntimeError, match="apply_tile_dev: unknown op kind: 3q"):
        _OpBatch([("3q", 1, 2, 3, np.eye(8))], 0)
    with pytest.raises(RuntimeError, match=r"apply_tile_dev: 1q expects"):
        _OpBatch([("1q", 1)], 0)
    with pytest.raises(RuntimeError, match="U must be a 2x2 matrix"):
        _OpBatch([("1q", 1, np.eye(3))], 0)


@pytest.mark.parametrize("n,seed", [(13, 0), (16, 1)])
def test_plan_emulation_adversarial_angles(native_lib, n, seed):
    # rotations whose cosine or sine nearly vanishes: the per-pass scalar extraction keeps the
    # complex64 state inside the single-precision range (no overflow, no underflow)
    from tests.cases import adversarial_angles
    qc = adversarial_angles(n, 12, seed)
    psi, _, _ = _emulate(qc, 0)
    assert np.all(np.isfinite(psi))
    assert O.infidelity(O.simulate(qc), psi) <= 1e-5
    assert abs(np.vdot(psi.astype(np.complex128), psi).real - 1.0) <= 1e-4
