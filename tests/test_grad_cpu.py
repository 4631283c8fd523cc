"""Host-side checks of the jit gradient's reverse program (no GPU): the program over the stacked
state psi (+) H psi, interpreted on the host with the gradient terms where the specialised
kernels take them (fixed-bit Z terms at their phase's start) and weighted by the scalars the
extraction took out before each term, must give the FP64 adjoint gradient of the oracle
(oracle/statevector.py adjoint_gradient, the restatement of the reverse sweep)."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.adjoint import ParamCircuit, ParamGate, grad_emulate
from frontierlabproject_b200.circuit import QuantumCircuit
from oracle import statevector as O


def _mixed(n, layers, seed, zero_every=0):
    """Rotations about X, Y and Z (some angles exactly 0 or near pi), CX / CZ between random
    pairs and fixed H / S gates; the same circuit as a ParamCircuit and a QuantumCircuit."""
    rng = np.random.default_rng(seed)
    pc = ParamCircuit(n)
    qc = QuantumCircuit(n)
    th = []
    for layer in range(layers):
        for q in range(n):
            name = ("rx", "ry", "rz")[int(rng.integers(3))]
            t = float(rng.uniform(-np.pi, np.pi))
            if zero_every and len(th) % zero_every == 0:
                t = 0.0
            if len(th) % 11 == 5:
                t = np.pi - 1e-7
            pc.gates.append(ParamGate(name, (q,), len(th)))
            getattr(qc, name)(t, q)
            th.append(t)
        for _ in range(n // 2):
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            name = ("cx", "cz")[int(rng.integers(2))]
            pc.gates.append(ParamGate(name, (a, b)))
            getattr(qc, name)(a, b)
        q = int(rng.integers(n))
        if layer % 2:
            pc.gates.append(ParamGate("h", (q,)))
            qc.h(q)
        else:
            pc.gates.append(ParamGate("s", (q,)))
            qc.s(q)
    pc.num_params = len(th)
    return pc, np.array(th), qc


def _check(pc, th, qc, a, b, tol=2e-5):
    E_ref, g_ref = O.adjoint_gradient(qc, a, b)
    psi = O.simulate(qc)
    lam = O.zz_x_apply(psi, a, b)
    g = grad_emulate(pc, th, psi.astype(np.complex64), lam.astype(np.complex64))
    assert g.shape == g_ref.shape
    assert np.linalg.norm(g - g_ref) <= tol * np.linalg.norm(g_ref)
    return g, g_ref


@pytest.mark.parametrize("n,L,seed", [(10, 3, 0), (12, 2, 1)])
def test_hea_reverse_program_matches_oracle(native_lib, n, L, seed):
    rng = np.random.default_rng(seed)
    th = rng.uniform(-np.pi, np.pi, 2 * n * L)
    a, b = C.hea_observable(n, seed + 1)
    _check(ParamCircuit.hea(n, L), th, C.hea_ansatz(n, L, th), a, b)


@pytest.mark.parametrize("seed", [2, 3])
def test_mixed_rotations_zero_and_near_pi_angles(native_lib, seed):
    n = 11
    pc, th, qc = _mixed(n, 4, seed, zero_every=7)
    a, b = C.hea_observable(n, seed)
    _check(pc, th, qc, a, b)


def test_shared_parameter_slots_add_up(native_lib):
    # two rotations reading the same parameter: their terms add into one slot
    n = 10
    pc = ParamCircuit(n)
    qc = QuantumCircuit(n)
    th = np.array([0.7, -1.3])
    for q in range(n):
        pc.gates.append(ParamGate("ry", (q,), 0))
        qc.ry(th[0], q)
    for q in range(n - 1):
        pc.gates.append(ParamGate("cz", (q, q + 1)))
        qc.cz(q, q + 1)
    for q in range(n):
        pc.gates.append(ParamGate("rx", (q,), 1))
        qc.rx(th[1], q)
    pc.num_params = 2
    a, b = C.hea_observable(n, 4)
    E_ref, g_each = O.adjoint_gradient(qc, a, b)
    psi = O.simulate(qc)
    lam = O.zz_x_apply(psi, a, b)
    g = grad_emulate(pc, th, psi.astype(np.complex64), lam.astype(np.complex64))
    want = np.array([g_each[:n].sum(), g_each[n:].sum()])
    assert np.allclose(g, want, rtol=2e-5, atol=2e-6)


def test_structure_checks(native_lib):
    pc = ParamCircuit(10, [ParamGate("cz", (0, 1), 0)], 1)
    with pytest.raises(ValueError):
        grad_emulate(pc, [0.1], np.zeros(1024, np.complex64), np.zeros(1024, np.complex64))


def test_reverse_program_kernels_compile_without_spills(native_lib):
    import ctypes
    from frontierlabproject_b200 import _native as N
    from frontierlabproject_b200.adjoint import AdjOps
    n = 14
    pc, th, _ = _mixed(n, 3, 5, zero_every=9)
    tab = AdjOps(pc)  # owns the matrices the op table points to
    ops = tab.update(th)
    sw = ctypes.c_int()
    log = ctypes.create_string_buffer(1 << 20)
    rc = N.lib().qs_grad_jit_check(n, ops.ctypes.data, len(ops), pc.num_params, None, ctypes.byref(sw), log,
                                   len(log))
    err = N.lib().qs_last_error()
    if rc != 0 and b"NVRTC" in err and b"not found" in err:
        pytest.skip("NVRTC unavailable")
    assert rc == 0, err.decode()
    assert sw.value >= 1
    text = log.value.decode()
    assert "registers" in text
    for line in text.splitlines():
        if "spill stores" in line:
            assert int(line.split("bytes spill stores")[0].split(",")[-1].strip()) == 0, line


def test_gradient_entry_points_validate_ops(native_lib):
    import ctypes
    from frontierlabproject_b200 import _native as N
    from frontierlabproject_b200.adjoint import AdjOps
    n = 10
    pc = ParamCircuit(n, [ParamGate("ry", (0,), 0), ParamGate("cz", (0, 1))], 1)
    tab = AdjOps(pc)  # owns the matrices the op table points to
    ops = tab.update([0.3])
    z = np.zeros(1 << n, np.complex64)
    g = np.zeros(1)

    def emulate(o, nq=n, npar=1):
        return N.lib().qs_grad_emulate(nq, o.ctypes.data, len(o), npar, None, z.ctypes.data, z.ctypes.data,
                                       g.ctypes.data)

    assert emulate(ops) == 0
    bad = ops.copy()
    bad[0]["q0"] = n
    assert emulate(bad) == N.QS_ERR_INVALID and b"invalid q0" in N.lib().qs_last_error()
    bad = ops.copy()
    bad[0]["grad_index"] = 1
    assert emulate(bad) == N.QS_ERR_INVALID and b"grad_index" in N.lib().qs_last_error()
    bad = ops.copy()
    bad[1]["gen"] = 3
    assert emulate(bad) == N.QS_ERR_INVALID and b"two-qubit" in N.lib().qs_last_error()
    bad = ops.copy()
    bad[1]["q1"] = 0
    assert emulate(bad) == N.QS_ERR_INVALID and b"q0/q1" in N.lib().qs_last_error()
    assert emulate(ops, nq=9) == N.QS_ERR_INVALID
    h = ctypes.c_void_p()
    assert N.lib().qs_grad_create(9, ops.ctypes.data, len(ops), 1, None, ctypes.byref(h)) == N.QS_ERR_INVALID
    assert not h.value
