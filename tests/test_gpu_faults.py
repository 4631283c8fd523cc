"""Failure detection on the GPU without a GPU fault.

* Bounded device waits: the limit of every wait of a state's kernels is a config field.  Set
  to 1 ns, the grid barriers of a cooperative multi-pass launch and the dependency waits of a
  batch launch run out on purpose (nothing else is wrong: the waits would end by themselves);
  the kernel sets its error word and returns, the call reports QS_ERR_DEVICE with the wait
  named, and the same state / a new batch then runs correctly with the default limit.
* Allocation failures: the library's k-th next allocation is made to fail on the host
  (qs_debug_fail_alloc); the call returns a clean CUDA out-of-memory error and frees what it
  had already allocated.
"""
import ctypes

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import run_custom_backend
from frontierlabproject_b200.batch import BatchedAdjoint, BatchShape, emulate, hea_batch
from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
from frontierlabproject_b200.transpiler import tile_circuit
from oracle import statevector as O

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_cooperative_barrier_wait_expires_and_state_recovers():
    n = 22
    qc = C.random_layered(n, 20, 4)
    _, plan = tile_circuit(qc, 16)
    sv = StatevectorF32(n)
    sv.set_config(wait_limit_ns=1)
    assert sv.get_config()["wait_limit_ns"] == 1
    with pytest.raises(RuntimeError, match="grid barrier wait expired"):
        run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="cooperative", sv=sv)
    # the error word was read and cleared; the C ABI status of a fresh occurrence is QS_ERR_DEVICE
    sv.reset()
    from frontierlabproject_b200.qgpusim_cuda import _OpBatch
    from tests.cases import ops_of
    b = _OpBatch(ops_of(qc), 0)
    N.call("qs_apply_tile", sv._h, b.ptr, len(b), N.MODES["cooperative"])
    rc = N.lib().qs_synchronize(sv._h)
    assert rc == N.QS_ERR_DEVICE
    assert b"grid barrier wait expired" in N.lib().qs_last_error()
    # default limit again: the same state object gives the right answer
    sv.set_config(wait_limit_ns=0)
    assert sv.get_config()["wait_limit_ns"] == 20 * 10 ** 9
    psi, _ = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="cooperative", sv=sv,
                                logical_order=True)
    assert O.infidelity(O.simulate_c(qc), psi) <= 1e-5


def test_batch_dependency_wait_expires_then_runs():
    insts = hea_batch(3, n_range=(17, 18), l_range=(3, 3), seed=8)
    shape = BatchShape(m=12, small_max=12, chunk=1, wait_limit_ns=1)
    b = BatchedAdjoint(insts, shape)
    b.run()
    with pytest.raises(RuntimeError, match="dependency wait"):
        b.results()
    ok = BatchedAdjoint(insts, BatchShape(m=12, small_max=12, chunk=1))
    E, G = ok.energies_and_grads()
    E_e, G_e = emulate(insts, BatchShape(m=12, small_max=12, chunk=1))
    np.testing.assert_allclose(E, E_e, rtol=1e-5, atol=1e-5)
    for g, ge in zip(G, G_e):
        assert np.linalg.norm(g - ge) <= 1e-5 * np.linalg.norm(ge)


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_state_creation_allocation_failure_frees_everything(k):
    L = N.lib()
    before = _free_bytes()
    h = ctypes.c_void_p()
    L.qs_debug_fail_alloc(k)
    try:
        rc = L.qs_create(24, N.QS_C64, ctypes.byref(h))
    finally:
        L.qs_debug_fail_alloc(0)
    assert rc == N.QS_ERR_CUDA
    assert b"out of memory" in L.qs_last_error()
    assert not h.value
    assert abs(_free_bytes() - before) < (64 << 20)  # the 128 MiB state was released
    sv = StatevectorF32(24)  # allocation works again
    assert sv.norm_squared() == pytest.approx(1.0)


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_batch_creation_allocation_failure_frees_everything(k):
    insts = hea_batch(4, n_range=(16, 18), l_range=(2, 3), seed=5)
    before = _free_bytes()
    N.lib().qs_debug_fail_alloc(k)
    try:
        with pytest.raises(RuntimeError, match="out of memory"):
            BatchedAdjoint(insts, BatchShape(m=12, small_max=12))
    finally:
        N.lib().qs_debug_fail_alloc(0)
    assert abs(_free_bytes() - before) < (16 << 20)
    E, _ = BatchedAdjoint(insts, BatchShape(m=12, small_max=12)).energies_and_grads()
    assert np.all(np.isfinite(E))


def test_sampling_allocation_failure_is_clean():
    sv = StatevectorF32(16)
    sv.apply_tile_cooperative([("1q", q, np.array([[1, 1], [1, -1]]) / np.sqrt(2)) for q in range(16)])
    sv.synchronize()
    for k in (1, 2):
        N.lib().qs_debug_fail_alloc(k)
        try:
            with pytest.raises(RuntimeError, match="out of memory"):
                sv.sample(1000)
        finally:
            N.lib().qs_debug_fail_alloc(0)
    idx = sv.sample(1000, seed=3)
    assert idx.size == 1000 and np.all(np.diff(idx.astype(np.int64)) >= 0)


def _grad_case(n=14, L=2, seed=3):
    from frontierlabproject_b200.adjoint import AdjOps, ParamCircuit
    pc = ParamCircuit.hea(n, L)
    th = np.random.default_rng(seed).uniform(-np.pi, np.pi, pc.num_params)
    a, b = C.hea_observable(n, seed)
    tab = AdjOps(pc)  # owns the matrices the op table points to
    return pc, th, a, b, tab, tab.update(th)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_gradient_handle_allocation_failure_frees_everything(k):
    pc, th, a, b, tab, ops = _grad_case()
    L = N.lib()
    before = _free_bytes()
    h = ctypes.c_void_p()
    L.qs_debug_fail_alloc(k)
    try:
        rc = L.qs_grad_create(pc.num_qubits, ops.ctypes.data, len(ops), pc.num_params, None, ctypes.byref(h))
    finally:
        L.qs_debug_fail_alloc(0)
    assert rc == N.QS_ERR_CUDA
    assert b"out of memory" in L.qs_last_error()
    assert not h.value
    assert abs(_free_bytes() - before) < (16 << 20)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_gradient_run_allocation_failure_then_runs(k):
    # the k-th allocation of the first run (program buffers, staging, term array) fails: a clean
    # error, and the same handle then gives the oracle's gradient
    pc, th, a, b, tab, ops = _grad_case()
    L = N.lib()
    h = ctypes.c_void_p()
    N.call("qs_grad_create", pc.num_qubits, ops.ctypes.data, len(ops), pc.num_params, None, ctypes.byref(h))
    try:
        E = ctypes.c_double()
        G = np.zeros(pc.num_params)
        L.qs_debug_fail_alloc(k)
        try:
            rc = L.qs_grad_run(h, ops.ctypes.data, len(ops), a.ctypes.data, b.ctypes.data, ctypes.byref(E),
                               G.ctypes.data)
        finally:
            L.qs_debug_fail_alloc(0)
        if rc != 0:
            assert rc == N.QS_ERR_CUDA
            assert b"out of memory" in L.qs_last_error()
        N.call("qs_grad_run", h, ops.ctypes.data, len(ops), a.ctypes.data, b.ctypes.data, ctypes.byref(E),
               G.ctypes.data)
        E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(pc.num_qubits, 2, th), a, b)
        assert abs(E.value - E_ref) <= 1e-5 * max(1.0, abs(E_ref))
        assert np.linalg.norm(G - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    finally:
        L.qs_grad_destroy(h)
