"""Device measurement sampling (qs_sample, run_custom_backend task="sampling") against |psi|^2."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import run_custom_backend
from frontierlabproject_b200.qgpusim_cuda import Statevector, StatevectorF32
from frontierlabproject_b200.transpiler import tile_circuit
from oracle import statevector as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cls,n", [(StatevectorF32, 10), (Statevector, 11), (StatevectorF32, 14)])
def test_sample_distribution(cls, n):
    rng = np.random.default_rng(n)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    sv = cls(n)
    sv.from_numpy(psi)
    shots = 400_000
    idx = sv.sample(shots, seed=5)
    assert idx.size == shots and np.all(np.diff(idx.astype(np.int64)) >= 0)
    assert int(idx.max()) < (1 << n)
    freq = np.bincount(idx.astype(np.int64), minlength=1 << n) / shots
    p = np.abs(psi) ** 2
    tv = 0.5 * np.abs(freq - p).sum()
    # total variation of an exact multinomial sample: about sqrt(2^n / (2 pi shots))
    assert tv < 3 * np.sqrt((1 << n) / (2 * np.pi * shots))
    # same seed, same indices; other seed, other indices
    assert np.array_equal(sv.sample(shots, seed=5), idx)
    assert not np.array_equal(sv.sample(shots, seed=6), idx)


def test_sample_ghz_and_basis_states():
    n = 20
    qc = C.ghz_chain(n)
    _, plan = tile_circuit(qc, 14)
    sv = StatevectorF32(n)
    run_custom_backend(qc, plan, "statevector", use_float32=True, sv=sv)
    counts = sv.sample_counts(100_000, seed=1)
    assert set(counts) <= {"0" * n, "1" * n}
    assert abs(counts["0" * n] - 50_000) < 1_000
    sv.reset()
    assert set(sv.sample(1000, seed=2).tolist()) == {0}
    assert sv.sample(0).size == 0


def test_run_custom_backend_sampling_task_in_logical_order():
    # a circuit whose last tile leaves a non-identity layout: counts are keyed by circuit qubits
    n = 13
    qc = C.random_layered(n, 6, 3)
    _, plan = tile_circuit(qc, 8)
    psi, met = run_custom_backend(qc, plan, "sampling", shots=200_000, use_float32=True)
    ref = O.simulate(qc)
    p = np.abs(ref) ** 2
    freq = np.zeros(1 << n)
    for key, c in met["counts"].items():
        freq[int(key, 2)] = c / 200_000
    assert 0.5 * np.abs(freq - p).sum() < 3 * np.sqrt((1 << n) / (2 * np.pi * 200_000))
