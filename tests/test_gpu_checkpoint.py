"""Checkpoint / resume of a tile-executor run: the state saved after some tiles (amplitudes in
the physical layout of the last tile, with that layout), loaded into a new state object, and the
remaining tiles run there give the same result as the uninterrupted run."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import fuse_tile_ops, tile_ops_for
from frontierlabproject_b200.qgpusim_cuda import Statevector, StatevectorF32
from frontierlabproject_b200.transpiler import tile_circuit

pytestmark = pytest.mark.gpu


def _run(sv, qc, tiles, layout, dtype):
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    for t in tiles:
        if list(t.layout) != layout:
            sv.permute(layout, t.layout)
            layout = list(t.layout)
        ops = fuse_tile_ops(tile_ops_for(t, qmap, dtype))
        if ops:
            sv.apply_tile_graphed(ops)
    return layout


@pytest.mark.parametrize("cls,dtype,tol", [(StatevectorF32, np.complex64, 0.0), (Statevector, np.complex128, 0.0)])
def test_save_load_resume(tmp_path, cls, dtype, tol):
    qc = C.random_layered(16, 12, 7)
    _, plan = tile_circuit(qc, 10)
    k = len(plan) // 2
    full = cls(16)
    lay_full = _run(full, qc, plan, list(range(16)), dtype)
    want = full.to_numpy()
    first = cls(16)
    lay = _run(first, qc, plan[:k], list(range(16)), dtype)
    path = str(tmp_path / "ckpt.npz")
    first.save(path, lay)
    resumed, lay2 = cls.load(path)
    assert lay2 == lay
    lay_end = _run(resumed, qc, plan[k:], lay2, dtype)
    assert lay_end == lay_full
    got = resumed.to_numpy()
    assert np.max(np.abs(got - want)) <= 1e-6 if dtype == np.complex64 else np.max(np.abs(got - want)) <= 1e-13
    with pytest.raises(RuntimeError, match="does not match"):
        (Statevector if cls is StatevectorF32 else StatevectorF32)(16).restore(path)
