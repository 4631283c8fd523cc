"""The drop-in boundary seen from the reference's side (no GPU needed).

The reference's ``run_custom_backend`` native branch (qgpusim/backends/custom/backend.py:405-522)
drives its native extension through a fixed set of calls: ``Statevector(n)`` /
``StatevectorF32(n)``, ``permute(layout_old, layout_new)``, ``apply_tile_cooperative /
apply_tile_graphed / apply_tile_dev(ops)`` with ``('1q', q, U_dev)`` / ``('2q', q0, q1, U_dev)``
tuples of CuPy matrices, ``synchronize()`` and ``to_numpy()``.  tests/golden/native_calls.*
record every such call for seven circuits, three tile modes and both precisions, made by the
reference's own code (tests/golden/make_golden.py).  Here:

* each recorded call binds to frontierlabproject_b200.qgpusim_cuda's classes (same names,
  same arguments) and every op list packs into the C ABI's qs_op array;
* with the reference checkout present, its native branch is run again against a spy built on
  this module's classes, and its calls equal the recorded ones.
The GPU replay of the same calls is tests/test_gpu_dropin.py.
"""
import inspect
import os

import numpy as np
import pytest

from frontierlabproject_b200 import qgpusim_cuda as Q
from tests.conftest import GOLDEN
from tests.golden import ref_harness as H

TRACE = (os.path.join(GOLDEN, "native_calls.json"), os.path.join(GOLDEN, "native_calls.npz"))


@pytest.fixture(scope="module")
def trace():
    return H.load_trace(*TRACE)


def _check_call(cls, c):
    name = c["call"]
    if name in ("Statevector", "StatevectorF32"):
        assert getattr(Q, name) is cls
        inspect.signature(cls.__init__).bind(None, c["num_qubits"])
        return
    meth = getattr(cls, name)
    sig = inspect.signature(meth)
    if name == "permute":
        sig.bind(None, c["layout_old"], c["layout_new"])
        assert sorted(c["layout_old"]) == sorted(c["layout_new"]) == list(range(len(c["layout_new"])))
    elif name.startswith("apply_tile_"):
        ops = [(op["kind"], *op["qubits"], op["U"]) for op in c["ops"]]
        sig.bind(None, ops)
        code = Q.N.QS_C64 if cls is Q.StatevectorF32 else Q.N.QS_C128
        for op in c["ops"]:  # the reference passes matrices in the state's precision
            assert op["U"].dtype == (np.complex64 if code == Q.N.QS_C64 else np.complex128)
        b = Q._OpBatch(ops, code)  # host packing into qs_op, as the call does before the ABI
        assert len(b) == len(ops)
    else:
        sig.bind(None)


def test_recorded_calls_bind_to_this_module(trace):
    assert len(trace) == 42
    modes = set()
    for t in trace:
        first = t["calls"][0]
        cls = getattr(Q, first["call"])
        assert (cls is Q.StatevectorF32) == t["f32"]
        names = [c["call"] for c in t["calls"]]
        assert names[-2:] == ["synchronize", "to_numpy"]
        assert any(n == {"cooperative": "apply_tile_cooperative", "graphed": "apply_tile_graphed",
                         "sequential": "apply_tile_dev"}[t["mode"]] for n in names)
        for c in t["calls"]:
            _check_call(cls, c)
        modes.add(t["mode"])
    assert modes == {"cooperative", "graphed", "sequential"}


def _spy_module(calls):
    """A native-extension stand-in whose classes are this module's classes' signatures:
    each call is bound and checked as above, then recorded like the fixture generator does."""
    rec = H.recording_module(calls)

    def checked(cls_name):
        base = getattr(rec, cls_name)
        real = getattr(Q, cls_name)

        class Spy(base):
            def __init__(self, num_qubits):
                inspect.signature(real.__init__).bind(None, num_qubits)
                super().__init__(num_qubits)

        for meth in ("permute", "apply_tile_cooperative", "apply_tile_graphed", "apply_tile_dev", "synchronize",
                     "to_numpy"):
            def wrap(m=meth):
                inner = getattr(base, m)

                def f(self, *a, **k):
                    inspect.signature(getattr(real, m)).bind(None, *a, **k)
                    return inner(self, *a, **k)
                return f
            setattr(Spy, meth, wrap())
        Spy.__name__ = cls_name
        return Spy

    rec.Statevector = checked("Statevector")
    rec.StatevectorF32 = checked("StatevectorF32")
    return rec


def test_reference_native_branch_against_this_module(trace):
    root = H.reference_root()
    if root is None:
        pytest.skip("reference checkout not present")
    passes = H.import_passes(root)
    from tests.cases import BUILDERS, nl_of
    done = 0
    for t in trace:
        if t["mode"] != "graphed" and done >= 6:
            continue
        qc = BUILDERS[t["case"]]()
        plan = H.reference_plan(passes, qc, nl_of(t["case"]))
        calls = []
        backend = H.import_native_branch(root, _spy_module(calls))
        backend.clear_gate_cache()
        backend.run_custom_backend(qc, plan, "statevector", use_float32=t["f32"], tile_mode=t["mode"])
        assert [c["call"] for c in calls] == [c["call"] for c in t["calls"]]
        for got, want in zip(calls, t["calls"]):
            for key in ("num_qubits", "layout_old", "layout_new"):
                assert got.get(key) == want.get(key)
            if "ops" in want:
                assert len(got["ops"]) == len(want["ops"])
                for a, b in zip(got["ops"], want["ops"]):
                    assert a["kind"] == b["kind"] and a["qubits"] == b["qubits"]
                    np.testing.assert_array_equal(a["U"], b["U"])
                _check_call(getattr(Q, calls[0]["call"]), got)
        done += 1
    assert done >= 6
