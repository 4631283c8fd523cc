"""The jit adjoint gradient on the GPU: the forward tile and the reverse program over the stacked
state psi (+) H psi, both run by plan-time specialised kernels, against the FP64 oracle adjoint
(oracle/statevector.py adjoint_gradient) and the host interpretation of the same program."""
import ctypes

import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from oracle import statevector as O
from tests.test_grad_cpu import _mixed

pytestmark = pytest.mark.gpu


def _rel(g, ref):
    return np.linalg.norm(g - ref) / np.linalg.norm(ref)


@pytest.mark.parametrize("n,L,seed", [(14, 3, 0), (16, 2, 1)])
def test_hea_matches_fp64_oracle(n, L, seed):
    from frontierlabproject_b200.adjoint import AdjointEngine, ParamCircuit
    rng = np.random.default_rng(seed)
    th = rng.uniform(-np.pi, np.pi, 2 * n * L)
    a, b = C.hea_observable(n, seed + 1)
    E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
    eng = AdjointEngine(n, f32=True, method="jit")
    E, g = eng.energy_and_grad(ParamCircuit.hea(n, L), th, a, b)
    assert abs(E - E_ref) <= 1e-5 * max(1.0, abs(E_ref))
    assert _rel(g, g_ref) <= 1e-5
    info = eng.info()
    assert info["reverse_sweeps"] >= 1 and info["terms"] == 2 * n * L


@pytest.mark.parametrize("seed", [2, 3])
def test_mixed_rotations_zero_and_near_pi_angles(seed):
    from frontierlabproject_b200.adjoint import AdjointEngine
    n = 14
    pc, th, qc = _mixed(n, 5, seed, zero_every=7)
    a, b = C.hea_observable(n, seed)
    E_ref, g_ref = O.adjoint_gradient(qc, a, b)
    E, g = AdjointEngine(n, f32=True, method="jit").energy_and_grad(pc, th, a, b)
    assert abs(E - E_ref) <= 1e-5 * max(1.0, abs(E_ref))
    assert _rel(g, g_ref) <= 1e-5


def test_parameter_updates_reuse_plans_and_kernels():
    from frontierlabproject_b200.adjoint import AdjointEngine, ParamCircuit, grad_emulate
    n, L = 15, 3
    pc = ParamCircuit.hea(n, L)
    a, b = C.hea_observable(n, 7)
    eng = AdjointEngine(n, f32=True, method="jit")
    rng = np.random.default_rng(11)
    for it in range(3):
        th = rng.uniform(-np.pi, np.pi, pc.num_params)
        E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
        E, g = eng.energy_and_grad(pc, th, a, b)
        assert _rel(g, g_ref) <= 1e-5, it
        assert abs(eng.energy(pc, th, a, b) - E) <= 1e-6 * max(1.0, abs(E))
        # the kernels' terms equal the host interpretation of the same program
        psi = O.simulate(C.hea_ansatz(n, L, th))
        ge = grad_emulate(pc, th, psi.astype(np.complex64), O.zz_x_apply(psi, a, b).astype(np.complex64))
        assert _rel(g, ge) <= 1e-5
    st = eng.info()
    assert st["graph_replays"] + st["graph_builds"] >= 3


def test_structure_change_is_rejected():
    from frontierlabproject_b200 import _native as N
    from frontierlabproject_b200.adjoint import AdjOps, ParamCircuit
    n = 12
    pc = ParamCircuit.hea(n, 2)
    th = np.zeros(pc.num_params)
    tab = AdjOps(pc)  # owns the matrices the op table points to
    ops = tab.update(th)
    h = ctypes.c_void_p()
    N.call("qs_grad_create", n, ops.ctypes.data, len(ops), pc.num_params, None, ctypes.byref(h))
    try:
        tab1 = AdjOps(ParamCircuit.hea(n, 1))
        other = tab1.update(np.zeros(2 * n))
        a, b = C.hea_observable(n, 0)
        E = ctypes.c_double()
        G = np.zeros(pc.num_params)
        rc = N.lib().qs_grad_run(h, other.ctypes.data, len(other), a.ctypes.data, b.ctypes.data, ctypes.byref(E),
                                 G.ctypes.data)
        assert rc == N.QS_ERR_INVALID
        assert b"structure" in N.lib().qs_last_error()
        # theta = 0 everywhere (identity rotations) still runs the planned program
        rc = N.lib().qs_grad_run(h, ops.ctypes.data, len(ops), a.ctypes.data, b.ctypes.data, ctypes.byref(E),
                                 G.ctypes.data)
        assert rc == 0, N.lib().qs_last_error()
        E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, 2, th), a, b)
        assert np.linalg.norm(G - g_ref) <= 1e-5 * max(1.0, np.linalg.norm(g_ref))
    finally:
        N.lib().qs_grad_destroy(h)


def test_circuit_without_gates_or_rotations():
    # no gate at all (psi = |0...0>), and fixed gates only: the energy, with empty / zero gradients
    from frontierlabproject_b200.adjoint import AdjointEngine, ParamCircuit, ParamGate
    from frontierlabproject_b200.circuit import QuantumCircuit
    n = 12
    a, b = C.hea_observable(n, 2)
    E, g = AdjointEngine(n, f32=True, method="jit").energy_and_grad(ParamCircuit(n, [], 0), [], a, b)
    psi0 = np.zeros(1 << n, dtype=np.complex128)
    psi0[0] = 1
    assert abs(E - O.energy(psi0, a, b)) <= 1e-6 and g.size == 0
    pc = ParamCircuit(n, [ParamGate("h", (q,)) for q in range(n)] + [ParamGate("cz", (0, 5))], 3)
    qc = QuantumCircuit(n)
    for q in range(n):
        qc.h(q)
    qc.cz(0, 5)
    E, g = AdjointEngine(n, f32=True, method="jit").energy_and_grad(pc, [0.1, 0.2, 0.3], a, b)
    assert abs(E - O.energy(O.simulate(qc), a, b)) <= 1e-5
    assert np.all(g == 0.0) and g.size == 3


@pytest.mark.parametrize("knobs", [{"jit_lr": 6}, {"m": 12, "k": 2}])
def test_plan_knobs_keep_the_gradient(knobs):
    # other register-bit counts and staging of the two programs: the same gradient
    from frontierlabproject_b200.adjoint import AdjointEngine, ParamCircuit
    n, L = 14, 3
    rng = np.random.default_rng(4)
    th = rng.uniform(-np.pi, np.pi, 2 * n * L)
    a, b = C.hea_observable(n, 5)
    E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
    eng = AdjointEngine(n, f32=True, method="jit")
    eng.set_config(**knobs)
    E, g = eng.energy_and_grad(ParamCircuit.hea(n, L), th, a, b)
    assert abs(E - E_ref) <= 1e-5 * max(1.0, abs(E_ref))
    assert _rel(g, g_ref) <= 1e-5
