"""Adjoint gradients on the GPU against the FP64 oracle, finite differences and parameter shift."""
import numpy as np
import pytest

from frontierlabproject_b200 import circuits as C
from oracle import statevector as O

pytestmark = pytest.mark.gpu


def _case(n, L, seed):
    from frontierlabproject_b200.adjoint import ParamCircuit
    rng = np.random.default_rng(seed)
    th = rng.uniform(-np.pi, np.pi, 2 * n * L)
    a, b = C.hea_observable(n, seed + 1)
    return ParamCircuit.hea(n, L), th, a, b


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("mode", ["graphed", "cooperative", "sequential"])
def test_adjoint_matches_fp64_oracle(f32, mode):
    from frontierlabproject_b200.adjoint import AdjointEngine
    n, L = 10, 3
    pc, th, a, b = _case(n, L, 0)
    E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
    eng = AdjointEngine(n, f32=f32, mode=mode)
    E, g = eng.energy_and_grad(pc, th, a, b)
    tol = 1e-5 if f32 else 1e-11
    assert abs(E - E_ref) <= tol * max(1.0, abs(E_ref))
    assert np.linalg.norm(g - g_ref) <= tol * np.linalg.norm(g_ref)


def test_adjoint_vs_finite_differences_and_param_shift():
    from frontierlabproject_b200.adjoint import AdjointEngine
    n, L = 12, 2
    pc, th, a, b = _case(n, L, 3)
    eng = AdjointEngine(n, f32=False)
    _, g = eng.energy_and_grad(pc, th, a, b)
    h = 1e-3
    for k in (0, 7, 23, 2 * n * L - 1):
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (eng.energy(pc, tp, a, b) - eng.energy(pc, tm, a, b)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k]))
    ps = eng.param_shift_grad(pc, th, a, b, params=[1, 5, 30])
    assert np.allclose(ps, g[[1, 5, 30]], atol=1e-11)


def test_c64_gradient_against_c128_n20():
    from frontierlabproject_b200.adjoint import AdjointEngine
    n, L = 20, 4
    pc, th, a, b = _case(n, L, 5)
    E32, g32 = AdjointEngine(n, f32=True).energy_and_grad(pc, th, a, b)
    E64, g64 = AdjointEngine(n, f32=False).energy_and_grad(pc, th, a, b)
    assert np.linalg.norm(g32 - g64) <= 1e-5 * np.linalg.norm(g64)
    assert abs(E32 - E64) <= 1e-5 * max(1.0, abs(E64))


def test_torch_autograd():
    import torch
    from frontierlabproject_b200.adjoint import AdjointEngine, expectation
    n, L = 8, 2
    pc, th, a, b = _case(n, L, 9)
    eng = AdjointEngine(n, f32=False)
    t = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    E = expectation(t, eng, pc, a, b)
    (2.0 * E).backward()
    E_ref, g_ref = O.adjoint_gradient(C.hea_ansatz(n, L, th), a, b)
    assert abs(E.item() - E_ref) < 1e-11
    assert np.allclose(t.grad.numpy(), 2.0 * g_ref, atol=1e-10)


@pytest.fixture(scope="module")
def config3():
    # the benchmark workload itself: n = 24, L = 20 (960 parameters, 1440 gates); the complex128
    # adjoint (per-gate reverse sweep) is the reference
    from frontierlabproject_b200.adjoint import AdjointEngine
    n, L = 24, 20
    pc, th, a, b = _case(n, L, 0)
    assert pc.num_params == 960
    eng64 = AdjointEngine(n, f32=False)
    E64, g64 = eng64.energy_and_grad(pc, th, a, b)
    return pc, th, a, b, eng64, E64, g64


@pytest.mark.parametrize("method", ["jit", "fused"])
def test_config3_full_size_c64_vs_c128(config3, method):
    # complex64 states with FP64 accumulation: the specialised-kernel program over the stacked
    # state (jit, the default at this size) and the batched persistent launch (fused)
    from frontierlabproject_b200.adjoint import AdjointEngine
    pc, th, a, b, _, E64, g64 = config3
    eng32 = AdjointEngine(24, f32=True, method=method)
    E32, g32 = eng32.energy_and_grad(pc, th, a, b)
    assert eng32.method == method
    assert np.linalg.norm(g32 - g64) <= 1e-5 * np.linalg.norm(g64)
    assert abs(E32 - E64) <= 1e-5 * max(1.0, abs(E64))
    assert AdjointEngine(24, f32=True).method == "jit"


def test_config3_c128_vs_finite_differences(config3):
    # the complex128 gradient against central finite differences (h = 1e-3) on 8 parameters
    pc, th, a, b, eng64, _, g64 = config3
    h = 1e-3
    for k in (0, 1, 137, 480, 481, 700, 958, 959):
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (eng64.energy(pc, tp, a, b) - eng64.energy(pc, tm, a, b)) / (2 * h)
        # central differences carry an O(h^2) truncation error: |E'''| h^2 / 6 ~ 1e-6 here
        assert abs(fd - g64[k]) <= 1e-5 * max(1.0, abs(g64[k])), (k, fd, g64[k])
