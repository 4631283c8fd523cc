"""The LQR tiler reproduces the reference's tile schedules exactly."""
import numpy as np
import pytest

from frontierlabproject_b200.transpiler import LazyQubitReordering, make_custom_pm, tile_circuit
from frontierlabproject_b200.transpiler.passes import _build_tile_layout
from tests.cases import BUILDERS, nl_of


def _record(qc, plan):
    pos = {(id(ins.operation), tuple(ins.qubits)): k for k, ins in enumerate(qc.data)}
    return [{"tile_idx": t.tile_idx, "logical_qubits": list(t.logical_qubits), "layout": list(t.layout),
             "gates": [pos[(id(g.op), tuple(g.qargs))] for g in t.gates]} for t in plan]


@pytest.mark.parametrize("native", [False, True], ids=["python", "native"])
@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_schedule_matches_reference(name, native, schedules):
    qc = BUILDERS[name]()
    nL = nl_of(name)
    _, plan = tile_circuit(qc, nL, native=native)
    assert _record(qc, plan) == schedules[name]["tiles"]


@pytest.mark.parametrize("n,depth,nL,seed", [(12, 10, 3, 1), (16, 20, 6, 2), (20, 30, 14, 3), (9, 15, 1, 4),
                                             (24, 12, 24, 5), (30, 40, 20, 6)])
def test_native_tiler_equals_python(n, depth, nL, seed):
    # same tiles, same gates per tile, same mapping sets (forced tiles included at small nL)
    from frontierlabproject_b200 import circuits as C
    qc = C.random_layered(n, depth, seed)
    qc.cx(0, n - 1)
    qc.swap(1, n // 2)
    out = {}
    for native in (False, True):
        pm, lqr = make_custom_pm(nL, native=native)
        tqc = pm.run(qc)
        plan = lqr.property_set["flat_tiling_plan"]
        sched = lqr.property_set["flat_tiling_schedule"]
        M = lqr.property_set["flat_tiling_mapping"]
        out[native] = (_record(qc, plan), [(id(nd.op), tuple(nd.qargs)) for nd in sched],
                       [sorted(M[nd]) for nd in sched], [ins.operation for ins in tqc.data])
    assert out[True] == out[False]


def test_native_tiler_rejects_bad_input(native_lib):
    import ctypes
    from frontierlabproject_b200 import _native as N
    masks = (ctypes.c_ulonglong * 1)(1 << 5)
    o, t, nt = (ctypes.c_int * 1)(), (ctypes.c_int * 1)(), ctypes.c_int()
    tm = (ctypes.c_ulonglong * 1)()
    with pytest.raises(RuntimeError, match="out of range"):
        N.call("qs_lqr_flat_tiling", 4, 2, masks, 1, o, t, tm, ctypes.byref(nt))
    with pytest.raises(RuntimeError, match="invalid argument"):
        N.call("qs_lqr_flat_tiling", 4, 0, masks, 1, o, t, tm, ctypes.byref(nt))


def test_published_tile_counts(schedules):
    # results/result.csv:6-8 (n=20) and :13-15 (n=25): 5 tiles / 4 reorders, 9 / 8
    for name, tiles in [("u_layers_n20_d16_s42_nL16_save", 5), ("u_layers_n25_d16_s42_nL16_save", 9)]:
        _, plan = tile_circuit(BUILDERS[name](), 16)
        assert len(plan) == tiles
        assert plan[-1].layout == list(range(plan[-1].layout.__len__()))  # forced all-qubit tile


def test_layout_and_local_map():
    assert _build_tile_layout([1, 4], 6) == [1, 4, 0, 2, 3, 5]
    _, plan = tile_circuit(BUILDERS["random_layered_n12_d8_s2_nL8"](), 8)
    for t in plan:
        assert t.logical_qubits == sorted(t.logical_qubits)
        assert t.layout[:len(t.logical_qubits)] == t.logical_qubits
        assert sorted(t.layout) == list(range(12))
        for q, i in t.global_to_local_map.items():
            assert t.layout[i] == q


def test_pass_manager_rewrites_in_schedule_order():
    qc = BUILDERS["qft_swaps_n9_nL5"]()
    pm, lqr = make_custom_pm(5)
    tqc = pm.run(qc)
    sched = lqr.property_set["flat_tiling_schedule"]
    assert [ins.operation for ins in tqc.data] == [n.op for n in sched]
    assert len(tqc.data) == len(qc.data)
    summ = LazyQubitReordering.summarize_tiling(sched, lqr.property_set["flat_tiling_mapping"])
    assert summ["num_tiles"] == len(lqr.property_set["flat_tiling_plan"])


def test_empty_and_tiny():
    from frontierlabproject_b200.circuit import QuantumCircuit
    _, plan = tile_circuit(QuantumCircuit(3), 2)
    assert plan == []
    qc = QuantumCircuit(1)
    qc.h(0)
    _, plan = tile_circuit(qc, 4)
    assert len(plan) == 1 and plan[0].layout == [0]


def _both(qc, nL):
    out = []
    for native in (False, True):
        _, plan = tile_circuit(qc, nL, native=native)
        out.append(_record(qc, plan))
    return out


@pytest.mark.parametrize("nL", [1, 2, 7, 8, 40])
def test_native_tiler_edge_sizes(nL):
    # nL = 1: every 2-qubit gate forces a tile; nL >= n: one tile; barriers (no unitary) included
    from frontierlabproject_b200 import circuits as C
    qc = C.random_layered(8, 6, 9)
    qc.barrier()
    qc.cx(7, 0)
    py, nat = _both(qc, nL)
    assert nat == py
    if nL >= 8:
        assert len(nat) == 1


def test_native_tiler_multi_qubit_targets():
    # a gate on three qubits (a barrier over three wires) goes through the same set logic
    from frontierlabproject_b200.circuit import QuantumCircuit
    qc = QuantumCircuit(6)
    for q in range(6):
        qc.h(q)
    qc.barrier(0, 2, 4)
    qc.cx(0, 5)
    qc.cx(1, 3)
    qc.barrier(1, 3, 5)
    qc.rz(0.3, 2)
    for nL in (2, 3, 4, 6):
        py, nat = _both(qc, nL)
        assert nat == py
