"""The reference's native branch replayed on the GPU through this module.

tests/golden/native_calls.* hold every call the reference's own ``run_custom_backend`` native
branch (qgpusim/backends/custom/backend.py:405-522) makes on its extension, for seven circuits,
three tile modes and both precisions.  Each trace is replayed call by call on
frontierlabproject_b200.qgpusim_cuda, with the gate matrices as device arrays exposing
``__cuda_array_interface__`` (torch CUDA tensors stand in for the reference's CuPy arrays), and
the ``to_numpy()`` result is compared with the reference executor's final state
(tests/golden/states.npz, complex128, physical layout of the last tile).
"""
import os

import numpy as np
import pytest

from frontierlabproject_b200 import qgpusim_cuda as Q
from oracle import statevector as O
from tests.conftest import GOLDEN
from tests.golden import ref_harness as H

pytestmark = pytest.mark.gpu

TRACE = (os.path.join(GOLDEN, "native_calls.json"), os.path.join(GOLDEN, "native_calls.npz"))


def _replay(t):
    import torch
    sv = None
    out = None
    keep = []
    for c in t["calls"]:
        name = c["call"]
        if name in ("Statevector", "StatevectorF32"):
            sv = getattr(Q, name)(c["num_qubits"])
        elif name == "permute":
            sv.permute(c["layout_old"], c["layout_new"])
        elif name.startswith("apply_tile_"):
            ops = []
            for op in c["ops"]:
                U = torch.from_numpy(np.ascontiguousarray(op["U"])).cuda()
                keep.append(U)
                ops.append((op["kind"], *op["qubits"], U))
            torch.cuda.synchronize()
            getattr(sv, name)(ops)
        elif name == "synchronize":
            sv.synchronize()
        elif name == "to_numpy":
            out = sv.to_numpy()
        else:
            raise AssertionError(f"unexpected call {name}")
    return out


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("mode", ["cooperative", "graphed", "sequential"])
def test_replay_reference_native_calls(mode, f32, golden_states):
    traces = [t for t in H.load_trace(*TRACE) if t["mode"] == mode and t["f32"] == f32]
    assert len(traces) == 7
    for t in traces:
        psi = _replay(t)
        ref = golden_states[t["case"]]
        assert psi.dtype == (np.complex64 if f32 else np.complex128)
        if f32:
            assert O.infidelity(ref, psi) <= 1e-5, t["case"]
            assert np.max(np.abs(psi.astype(np.complex128) - ref)) <= 1e-5, t["case"]
        else:
            assert np.max(np.abs(psi - ref)) <= 1e-12, t["case"]
