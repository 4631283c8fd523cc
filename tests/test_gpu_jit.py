"""Plan-time specialised pass kernels (NVRTC, graphed mode, complex64) against the oracle."""
import ctypes

import numpy as np
import pytest

from frontierlabproject_b200 import _native as N
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import run_custom_backend
from frontierlabproject_b200.qgpusim_cuda import StatevectorF32, _OpBatch
from frontierlabproject_b200.transpiler import tile_circuit
from oracle import statevector as O
from tests.cases import BUILDERS, ops_of
from tests.test_planner_cpu import _mixed


def test_jit_source_compiles_for_sm100a(native_lib):
    qc = _mixed(12, 3)
    b = _OpBatch(ops_of(qc), 0)
    sw = ctypes.c_int()
    log = ctypes.create_string_buffer(1 << 16)
    rc = native_lib.qs_jit_check(12, b.ptr, len(b), None, ctypes.byref(sw), log, len(log))
    if rc != 0 and b"NVRTC" in native_lib.qs_last_error() and b"not found" in native_lib.qs_last_error():
        pytest.skip("NVRTC unavailable")
    assert rc == 0, native_lib.qs_last_error().decode()
    assert sw.value >= 1
    # specialised kernels hold all amplitudes in registers: no local-memory spills
    text = log.value.decode()
    assert "registers" in text
    assert "0 bytes spill stores" in text and "bytes spill stores" in text
    for line in text.splitlines():
        if "spill stores" in line:
            assert line.strip().startswith("0 bytes stack frame") or " 0 bytes spill stores" in line, line


def _run_jit(qc, nl, blocks=2, packed=0, lr=5, **kw):
    _, plan = tile_circuit(qc, nl)
    sv = StatevectorF32(qc.num_qubits)
    sv.set_config(jit=1, jit_blocks=blocks, jit_packed=packed, jit_lr=lr)
    psi, met = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv, **kw)
    return psi, met, plan, sv


@pytest.mark.gpu
@pytest.mark.parametrize("blocks,packed", [(1, 0), (2, 0), (3, 0), (2, 1), (3, 1)])
@pytest.mark.parametrize("n", [9, 13, 16])
def test_jit_mixed_gates(n, blocks, packed):
    qc = _mixed(n, n + 1)
    psi, met, plan, sv = _run_jit(qc, max(4, n - 3), blocks, packed, logical_order=True)
    assert O.infidelity(O.simulate(qc), psi) <= 1e-5
    assert np.max(np.abs(psi - O.simulate(qc))) <= 1e-5
    assert sv.stats()["graph_builds"] >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["random_layered_n12_d8_s2_nL8", "qft_swaps_n9_nL5", "hea_n8_L3_nL5",
                                  "reference_random_n10_d4_s42_nL6"])
def test_jit_reference_executor_states(name, golden_states):
    qc = BUILDERS[name]()
    nl = int(name.split("_nL")[1].split("_")[0])
    psi, _, _, _ = _run_jit(qc, nl)
    assert O.infidelity(golden_states[name], psi) <= 1e-5


@pytest.mark.gpu
def test_jit_config0_n20_and_replay():
    # n=20 takes the specialised kernels by default; a second run replays the cached graph
    qc = C.random_layered(20, 20, 0)
    _, plan = tile_circuit(qc, 14)
    ref, _ = O.run_tile_plan(qc, plan, np.complex128)
    sv = StatevectorF32(20)
    for _ in range(2):
        psi, met = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv)
        assert O.infidelity(ref, psi) <= 1e-5
    st = sv.stats()
    assert st["graph_replays"] >= 1


@pytest.mark.gpu
def test_jit_parameter_change_reuses_kernels():
    # same structure, new angles: results follow the new angles (coefficients are data)
    n, L = 14, 3
    rng = np.random.default_rng(0)
    sv = StatevectorF32(n)
    sv.set_config(jit=1)
    a, b = C.hea_observable(n, 1)
    for trial in range(2):
        th = rng.uniform(-np.pi, np.pi, 2 * n * L)
        qc = C.hea_ansatz(n, L, th)
        _, plan = tile_circuit(qc, 10)
        psi, _ = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv,
                                    logical_order=True)
        assert O.infidelity(O.simulate(qc), psi) <= 1e-5


def _flip_frame_circuit(n, seed):
    """Many CX/CY/CU gates whose controls are high qubits (group or warp-index bits of the
    passes) onto low targets, followed in the same layer by 1q, SWAP, controlled and dense
    2q gates on those targets: exercises the bit-flip frame of the specialised kernels."""
    from frontierlabproject_b200.circuit import QuantumCircuit
    rng = np.random.default_rng(seed)
    qc = QuantumCircuit(n)
    lo = list(range(8))
    hi = list(range(n - 7, n))
    U = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))[0]
    for layer in range(10):
        for q in range(n):
            [qc.h, qc.sx, qc.x][q % 3](q) if (q + layer) % 2 else qc.rx(float(rng.uniform(0, 6.28)), q)
        for _ in range(6):
            qc.cx(int(rng.choice(hi)), int(rng.choice(lo)))
        a, b = rng.choice(lo, 2, replace=False)
        qc.cx(int(a), int(b))
        qc.rz(float(rng.uniform(0, 6.28)), int(b))
        a, b = rng.choice(lo, 2, replace=False)
        qc.swap(int(a), int(b))
        qc.h(int(a))
        qc.cy(int(rng.choice(hi)), int(rng.choice(lo)))
        a, b = rng.choice(lo, 2, replace=False)
        qc.crz(float(rng.uniform(0, 6.28)), int(a), int(b))
        qc.cp(float(rng.uniform(0, 6.28)), int(rng.choice(hi)), int(rng.choice(lo)))
        a, b = rng.choice(lo, 2, replace=False)
        qc.unitary(U, [int(a), int(b)])
        qc.ry(float(rng.uniform(0, 6.28)), int(a))
    return qc


@pytest.mark.gpu
@pytest.mark.parametrize("blocks,packed", [(2, 0), (3, 0), (2, 1)])
@pytest.mark.parametrize("n,seed", [(16, 1), (20, 2)])
def test_jit_flip_frame(n, seed, blocks, packed):
    qc = _flip_frame_circuit(n, seed)
    psi, _, _, _ = _run_jit(qc, n - 2, blocks, packed, logical_order=True)
    ref = O.simulate(qc)
    assert O.infidelity(ref, psi) <= 1e-5
    assert np.max(np.abs(psi - ref)) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("n", [21, 24])
def test_jit_teams_equal_single_team_bitwise(n):
    # the two-team schedule (three rotating buffers, many groups per block at n=24) runs the
    # same per-amplitude arithmetic as one team per block: identical bits
    qc = C.random_layered(n, 12, 5)
    psi2, _, _, _ = _run_jit(qc, n - 6, 2)
    psi3, _, _, sv = _run_jit(qc, n - 6, 3)
    assert sv.get_config()["jit_blocks"] == 3
    np.testing.assert_array_equal(psi3.view(np.uint32), psi2.view(np.uint32))
    assert abs(np.vdot(psi3.astype(np.complex128), psi3).real - 1.0) <= 1e-4


_DISK_PROBE = r"""
import json, sys
import numpy as np
sys.path.insert(0, ".")
from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.backend import run_custom_backend
from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
from frontierlabproject_b200.transpiler import tile_circuit
qc = C.random_layered(20, 6, 9)
_, plan = tile_circuit(qc, 14)
sv = StatevectorF32(20)
sv.set_config(jit=1)
psi, _ = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv)
st = sv.stats()
print(json.dumps({"modules": st["jit_modules"], "hits": st["jit_disk_hits"],
                  "sum": [float(np.real(psi).sum()), float(np.imag(psi).sum())]}))
"""


@pytest.mark.gpu
def test_jit_disk_cache_across_processes(tmp_path):
    # a second process finds every kernel module of the same program on disk and gets the same state
    import json
    import os
    import subprocess
    import sys
    from tests.conftest import REPO
    env = dict(os.environ, QSIM_JIT_CACHE=str(tmp_path / "jit"))
    outs = []
    for _ in range(2):
        r = subprocess.run([sys.executable, "-c", _DISK_PROBE], cwd=REPO, env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    assert outs[0]["modules"] >= 1 and outs[0]["hits"] == 0
    assert outs[1]["hits"] == outs[1]["modules"] == outs[0]["modules"]
    assert outs[1]["sum"] == outs[0]["sum"]
    assert any(p.endswith(".cubin") for p in os.listdir(tmp_path / "jit"))


@pytest.mark.gpu
def test_jit_async_generic_stand_in_then_specialised():
    # a new structure: the first run goes through the generic kernel while the specialised
    # kernels compile in the background; after qs_jit_wait the next run uses them; both exact
    qc = C.random_layered(20, 8, 31)
    _, plan = tile_circuit(qc, 14)
    ref = O.simulate(qc)
    sv = StatevectorF32(20)
    sv.set_config(jit=1, jit_async=1)
    assert sv.get_config()["jit_async"] == 1
    psi, _ = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv,
                                logical_order=True)
    st = sv.stats()
    assert st["jit_pending_flushes"] >= 1 and st["jit_modules"] == 0
    assert O.infidelity(ref, psi) <= 1e-5
    StatevectorF32.jit_wait()
    psi2, _ = run_custom_backend(qc, plan, "statevector", use_float32=True, tile_mode="graphed", sv=sv,
                                 logical_order=True)
    st = sv.stats()
    assert st["jit_modules"] >= 1 and st["jit_pending_flushes"] == 0
    assert O.infidelity(ref, psi2) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("blocks", [1, 2, 3])
@pytest.mark.parametrize("n", [16, 20])
def test_jit_six_register_bits(n, blocks):
    # 64 amplitudes per thread, 2^(m-6) threads per group: mixed gates and the bit-flip frame
    for qc in (_mixed(n, n + 3), _flip_frame_circuit(n, 4)):
        psi, _, _, sv = _run_jit(qc, n - 2, blocks, 0, 6, logical_order=True)
        assert sv.get_config()["jit_lr"] == 6
        ref = O.simulate(qc)
        assert O.infidelity(ref, psi) <= 1e-5
        assert np.max(np.abs(psi - ref)) <= 1e-5
