"""Full-size GHZ (n=32) and QFT (n=30, with swaps) through every tile mode at nL = 16, 20, 24.

The states are 32 GiB and 8 GiB (complex64), too large for a CPU simulation inside a test, so
they are checked on the device against closed forms: the GHZ chain gives
(|0..0> + |1..1>)/sqrt2; the QFT of a basis state |x> gives exp(2 pi i x y / N)/sqrt N at
index y.  Both are read after the state is permuted back to logical order, so the check also
covers every layout change of the tile schedule.  The closed forms themselves are pinned
against the oracle at small n by the CPU tests at the end of this file.
"""
import math

import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from frontierlabproject_b200.circuit import QuantumCircuit
from frontierlabproject_b200.transpiler import tile_circuit

MODES = ["cooperative", "graphed", "sequential"]
QFT_X = 0b101100111000111100001101010011  # basis state fed to the 30-qubit QFT


def qft_of_basis(n: int, x: int) -> QuantumCircuit:
    qc = QuantumCircuit(n)
    for b in range(n):
        if (x >> b) & 1:
            qc.x(b)
    src = C.qft(n, True)
    for ins in src.data:
        qc.append(ins.operation, [src.find_bit(q).index for q in ins.qubits])
    return qc


def qft_closed_form(n: int, x: int) -> np.ndarray:
    y = np.arange(1 << n, dtype=np.int64)
    return np.exp(2j * np.pi * ((x * y) % (1 << n)) / (1 << n)) / math.sqrt(1 << n)


def _run_logical(qc, nl, mode):
    """Run the tile schedule through ``run_custom_backend``'s steps, ending in logical order,
    and return the device state without copying 2^n amplitudes to the host."""
    from frontierlabproject_b200.backend import fuse_tile_ops, tile_ops_for
    from frontierlabproject_b200.qgpusim_cuda import StatevectorF32
    _, plan = tile_circuit(qc, nl)
    n = qc.num_qubits
    qmap = {q: qc.find_bit(q).index for q in qc.qubits}
    sv = StatevectorF32(n)
    apply = {"cooperative": sv.apply_tile_cooperative, "graphed": sv.apply_tile_graphed,
             "sequential": sv.apply_tile_dev}[mode]
    layout = list(range(n))
    for t in plan:
        if list(t.layout) != layout:
            sv.permute(layout, t.layout)
            layout = list(t.layout)
        ops = fuse_tile_ops(tile_ops_for(t, qmap, np.complex64))
        if ops:
            apply(ops)
    sv.permute(layout, list(range(n)))
    sv.synchronize()
    return sv


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("nl", [16, 20, 24])
def test_ghz_chain_n32(nl, mode):
    import torch
    sv = _run_logical(C.ghz_chain(32), nl, mode)
    v = sv.torch_view()
    h = 2 ** -0.5
    a0, a1 = v[0].item(), v[-1].item()
    nz = int((v.abs() > 1e-6).sum().item())
    del v, sv
    torch.cuda.empty_cache()
    assert abs(a0 - h) < 1e-6 and abs(a1 - h) < 1e-6
    assert nz == 2


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("nl", [16, 20, 24])
def test_qft_n30_basis_state(nl, mode):
    import torch
    n = 30
    sv = _run_logical(qft_of_basis(n, QFT_X), nl, mode)
    v = sv.torch_view()
    y = torch.arange(1 << n, device=v.device, dtype=torch.int64)
    phase = ((QFT_X * y) % (1 << n)).to(torch.float64).mul_(2 * math.pi / (1 << n))
    del y
    amp = 2 ** (-n / 2)
    err_re = (v.real.double() - amp * torch.cos(phase)).abs().max().item()
    err_im = (v.imag.double() - amp * torch.sin(phase)).abs().max().item()
    del phase, v, sv
    torch.cuda.empty_cache()
    # amplitudes are 3.05e-5; complex64 rounding over the 465 gates stays far below 1e-8
    assert max(err_re, err_im) < 1e-8


# ---- CPU: the closed forms above against the oracle ------------------------------------

@pytest.mark.parametrize("n", [3, 6, 9])
def test_qft_closed_form_matches_oracle(n):
    from oracle.statevector import simulate
    x = QFT_X & ((1 << n) - 1)
    psi = simulate(qft_of_basis(n, x))
    np.testing.assert_allclose(psi, qft_closed_form(n, x), atol=1e-12)


def test_ghz_closed_form_matches_oracle():
    from oracle.statevector import simulate
    psi = simulate(C.ghz_chain(10))
    want = np.zeros(1 << 10, complex)
    want[0] = want[-1] = 2 ** -0.5
    np.testing.assert_allclose(psi, want, atol=1e-12)
