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


def test_noalloc_rejects_programs_beyond_the_workspace():
    import torch
    n = 14
    dev = torch.zeros(1 << n, dtype=torch.complex64, device="cuda")
    ops = _ops(3, n) * 600  # far beyond the fixed 1 MiB program space
    batch = _OpBatch(ops, 0)
    rc = N.lib().qs_apply_ops_noalloc(ctypes.c_void_p(dev.data_ptr()), 0, n, batch.ptr, len(batch), None)
    assert rc != 0
    assert b"static workspace" in N.lib().qs_last_error()
