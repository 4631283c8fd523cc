"""The allocation-free entry point qs_apply_ops_noalloc, through the C ABI.

It serves callers that may not allocate device memory (their framework's allocator owns
the device memory, or they cannot afford the synchronisation of cudaMalloc/cudaFree): the
caller owns the state; the program and barrier words live in the library's fixed device
array.  Its results must equal those of the allocating entry point (qs_apply_tile,
cooperative mode) within the test tolerance, on two calls in a row (the shared array keeps
the previous call's contents, which must not leak into the next call).

This file is collected last so a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.qgpusim_cuda import Statevector, StatevectorF32, _OpBatch
from oracle import statevector as O
from tests.cases import ops_of

pytestmark = pytest.mark.gpu

TOL = {np.complex64: 1e-5, np.complex128: 1e-12}


def _ops(seed, n):
    qc = C.random_layered(n, 6, seed)
    qc.cz(0, n - 1)
    qc.swap(1, n - 2)
    qc.cp(0.4, 2, 5)
    return ops_of(qc)


@pytest.mark.parametrize("dt", [np.complex64, np.complex128])
def test_noalloc_matches_allocating_entry_point(dt):
    import torch
    n = 17
    code = 0 if dt == np.complex64 else 1
    rng = np.random.default_rng(11)
    psi0 = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dt)
    psi0 /= np.linalg.norm(psi0)
    # existing entry point: a library-owned state, cooperative tile mode
    sv = (StatevectorF32 if code == 0 else Statevector)(n)
    sv.from_numpy(psi0)
    # allocation-free entry point: a caller-owned device array
    dev = torch.from_numpy(psi0.copy()).cuda()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    oracle = psi0.astype(np.complex128)
    for call, seed in enumerate((1, 2)):  # two calls in a row
        ops = _ops(seed, n)
        sv.apply_tile_cooperative(ops)
        ref = sv.to_numpy()
        batch = _OpBatch(ops, code)
        rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(dev.data_ptr()), code, n, batch.ptr, len(batch),
                                          ctypes.c_void_p(stream))
        assert rc == 0, N.lib().qs_last_error().decode()
        got = dev.cpu().numpy()
        assert np.max(np.abs(got.astype(np.complex128) - ref)) <= TOL[dt], f"call {call + 1}"
        # and against the FP64 oracle (the reference's per-gate arithmetic)
        for op in ops:
            if op[0] == "1q":
                O.apply_1q(oracle, op[2], op[1])
            else:
                O.apply_2q(oracle, op[3], op[1], op[2])
        assert np.max(np.abs(got.astype(np.complex128) - oracle)) <= TOL[dt], f"call {call + 1} vs oracle"


def test_noalloc_rejects_programs_beyond_the_workspace():
    import torch
    n = 14
    dev = torch.zeros(1 << n, dtype=torch.complex64, device="cuda")
    ops = _ops(3, n) * 600  # far beyond the fixed 1 MiB program space
    batch = _OpBatch(ops, 0)
    rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(dev.data_ptr()), 0, n, batch.ptr, len(batch), None)
    assert rc != 0
    assert b"static workspace" in N.lib().qs_last_error()


def test_noalloc_rejects_unaligned_and_host_pointers():
    # checked on the host before anything is launched: the kernel moves 16-byte units
    import torch
    n = 14
    dev = torch.zeros((1 << n) + 1, dtype=torch.complex64, device="cuda")
    batch = _OpBatch(_ops(4, n), 0)
    rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(dev[1:].data_ptr()), 0, n, batch.ptr, len(batch), None)
    assert rc == N.QS_ERR_INVALID
    assert b"16-byte aligned" in N.lib().qs_last_error()
    host = np.zeros(1 << n, dtype=np.complex64)
    rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(host.ctypes.data), 0, n, batch.ptr, len(batch), None)
    assert rc == N.QS_ERR_INVALID
    assert b"qs_apply_ops_noalloc" in N.lib().qs_last_error()
    # op validation errors name this entry point
    bad = np.zeros(1, dtype=N.OP_DTYPE)
    bad["kind"] = 7
    rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(dev.data_ptr()), 0, n, bad.ctypes.data, 1, None)
    assert rc == N.QS_ERR_INVALID
    assert N.lib().qs_last_error().startswith(b"qs_apply_ops_noalloc: unknown op kind")
